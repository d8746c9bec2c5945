"""FP64 CPU oracle of the warm-start MLP -- TEST INFRASTRUCTURE ONLY.

Restates the network of rq_mlp_* (include/ruqu_cuda.h): in -> h1 -> h2 -> out,
ReLU after the hidden layers, mean-squared-error loss, flat parameter layout
W1 [h1 x in], b1, W2 [h2 x h1], b2, W3 [out x h2], b3.  With `mimic_bf16`
the inputs, weights, hidden activations and back-propagated gradients are
rounded to bfloat16 at exactly the points where the GPU feeds its BF16 tensor
cores, so the remaining differences are FP32-vs-FP64 accumulation only.
(The reference has no MLP; this oracle checks the GPU kernels' gradients.)
"""
import numpy as np


def bf16(x):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p, dims):
    i, h1, h2, o = dims
    k = 0
    out = []
    for r, c in ((h1, i), (1, h1), (h2, h1), (1, h2), (o, h2), (1, o)):
        out.append(np.asarray(p[k:k + r * c], dtype=np.float64).reshape(r, c) if r > 1 else
                   np.asarray(p[k:k + c], dtype=np.float64))
        k += r * c
    return out


def forward_backward(params, dims, x, t, mimic_bf16=True):
    """Returns (y, loss, flat gradient)."""
    W1, b1, W2, b2, W3, b3 = unpack(params, dims)
    r = bf16 if mimic_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    X = r(x)
    Z1 = X @ r(W1).T + b1
    H1 = np.maximum(Z1, 0)
    Z2 = r(H1) @ r(W2).T + b2
    H2 = np.maximum(Z2, 0)
    Y = r(H2) @ r(W3).T + b3
    B, O = t.shape
    d = Y - t
    loss = float(np.sum(d * d) / (B * O))
    dY = 2.0 * d / (B * O)
    gW3 = r(dY).T @ r(H2)
    gb3 = dY.sum(0)
    dH2 = r(dY) @ r(W3)
    dZ2 = np.where(Z2 > 0, dH2, 0.0)
    gW2 = r(dZ2).T @ r(H1)
    gb2 = dZ2.sum(0)
    dH1 = r(dZ2) @ r(W2)
    dZ1 = np.where(Z1 > 0, dH1, 0.0)
    gW1 = r(dZ1).T @ X
    gb1 = dZ1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return Y, loss, g
