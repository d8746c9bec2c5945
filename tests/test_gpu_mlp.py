"""Tensor-core (tcgen05) BF16 GEMM and the warm-start MLP (needs a GPU).

The GEMM is checked against an FP64 product of the same BF16-rounded inputs
(tolerance 2e-3 relative to the row norms: FP32 accumulation in a different
order); the MLP's forward pass and gradients against the FP64 oracle MLP.
"""
import ctypes as C

import numpy as np
import pytest

from ruqu_b200 import _capi

pytestmark = pytest.mark.gpu


def bf16_bits(x):
    """Round-to-nearest-even float32 -> bfloat16 bit patterns."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return b.astype(np.uint16)


def bf16_value(bits):
    return (bits.astype(np.uint32) << 16).view(np.float32)


def gemm(A, B):
    M, K = A.shape
    N = B.shape[0]
    a, b = bf16_bits(A), bf16_bits(B)
    out = np.empty((M, N), dtype=np.float32)
    rc = _capi.lib.rq_gemm_bf16(a.ctypes.data_as(C.POINTER(C.c_uint16)), b.ctypes.data_as(C.POINTER(C.c_uint16)),
                                M, N, K, out.ctypes.data_as(C.POINTER(C.c_float)))
    assert rc == 0, _capi.last_error()
    ref = bf16_value(a).astype(np.float64) @ bf16_value(b).astype(np.float64).T
    return out, ref


@pytest.mark.parametrize("M,N,K", [(128, 32, 16), (128, 64, 64), (256, 128, 288), (128, 256, 256), (384, 256, 80),
                                   (512, 32, 512)])
def test_gemm_bf16_matches_fp64(M, N, K):
    r = np.random.default_rng(M + N + K)
    A = r.normal(size=(M, K)).astype(np.float32)
    B = r.normal(size=(N, K)).astype(np.float32)
    out, ref = gemm(A, B)
    scale = np.sqrt(K) * 1.0
    assert np.max(np.abs(out - ref)) < 2e-3 * scale, float(np.max(np.abs(out - ref)))


def test_gemm_bf16_structure():
    """Identity and permutation operands land in the right rows and columns."""
    M, N, K = 128, 128, 128
    A = np.eye(M, K, dtype=np.float32) * np.arange(1, M + 1, dtype=np.float32)[:, None]
    perm = np.random.default_rng(0).permutation(K)
    B = np.eye(K, dtype=np.float32)[perm][:N]
    out, ref = gemm(A, B)
    assert np.array_equal(out, ref.astype(np.float32))


# ---------------------------------------------------------------- the MLP
from oracle import mlp as omlp   # noqa: E402
from ruqu_b200.warmstart import Mlp   # noqa: E402

DIMS = (325, 256, 256, 8)


def _blocks(flat):
    i, h1, h2, o = DIMS
    sizes = [h1 * i, h1, h2 * h1, h2, o * h2, o]
    out, k = [], 0
    for s in sizes:
        out.append(flat[k:k + s])
        k += s
    return out


def test_mlp_forward_and_gradients_match_oracle():
    net = Mlp(*DIMS, seed=3)
    p = net.get_params()
    r = np.random.default_rng(4)
    B = 200
    x = (r.random((B, DIMS[0])) < 0.1).astype(np.float32)       # sparse 0/1 adjacency features
    t = r.uniform(0, 1.5, size=(B, DIMS[3])).astype(np.float32)
    y = net.forward(x)
    y_ref, _, _ = omlp.forward_backward(p, DIMS, x, t, mimic_bf16=True)
    assert np.max(np.abs(y - y_ref)) < 1e-3 * (1 + np.max(np.abs(y_ref)))
    loss, g = net.gradients(x, t)
    _, loss_ref, g_ref = omlp.forward_backward(p, DIMS, x, t, mimic_bf16=True)
    assert abs(loss - loss_ref) < 1e-4 * (1 + loss_ref)
    for a, b in zip(_blocks(g), _blocks(g_ref)):
        assert np.linalg.norm(a - b) <= 2e-3 * (np.linalg.norm(b) + 1e-12), (np.linalg.norm(a - b), np.linalg.norm(b))
    # and against the unrounded FP64 network: BF16 storage error only
    _, _, g64 = omlp.forward_backward(p, DIMS, x, t, mimic_bf16=False)
    for a, b in zip(_blocks(g), _blocks(g64)):
        assert np.linalg.norm(a - b) <= 5e-2 * (np.linalg.norm(b) + 1e-12)


def test_mlp_training_reduces_loss():
    net = Mlp(*DIMS, seed=5)
    r = np.random.default_rng(6)
    n = 1024
    x = (r.random((n, DIMS[0])) < 0.1).astype(np.float32)
    proj = r.normal(size=(DIMS[0], DIMS[3])) * 0.3
    t = (np.tanh(x @ proj) + 1.0).astype(np.float32)
    l0, _ = net.gradients(x[:256], t[:256])
    last = net.train(x, t, batch=256, steps=300, lr=1e-3)
    l1, _ = net.gradients(x[:256], t[:256])
    assert last < 0.3 * l0 and l1 < 0.3 * l0, (l0, last, l1)
