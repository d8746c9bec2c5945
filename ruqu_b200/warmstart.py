"""Learned warm start for QAOA angles (rq_mlp_* of include/ruqu_cuda.h).

A small MLP maps a padded graph adjacency (upper triangle of a 26-node
adjacency matrix, 325 binary features, so graphs up to 26 nodes fit) to the
2p QAOA angles (gamma_1..gamma_p, beta_1..beta_p).  Its forward and backward
passes run on the GPU's BF16 tensor cores (tcgen05) with FP32 accumulation,
FP32 master weights and Adam on the device.  The reference has no learned
component; its run_qaoa starts every instance from gamma = beta = 0.5
(crates/ruqu-algorithms/src/qaoa.rs:221-222).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import lib
from .error import check

PAD_NODES = 26
FEATURES = PAD_NODES * (PAD_NODES - 1) // 2      # 325


def graph_features(n: int, edges) -> np.ndarray:
    """Upper triangle (i < j, row-major) of the adjacency matrix padded to PAD_NODES nodes."""
    if n > PAD_NODES:
        raise ValueError(f"graphs up to {PAD_NODES} nodes")
    a = np.zeros((PAD_NODES, PAD_NODES), dtype=np.float32)
    for u, v in edges:
        a[u, v] = a[v, u] = 1.0
    iu = np.triu_indices(PAD_NODES, 1)
    return a[iu]


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    def __init__(self, n_in: int = FEATURES, h1: int = 256, h2: int = 256, n_out: int = 8, seed: int = 0):
        self.dims = (n_in, h1, h2, n_out)
        h = C.c_void_p()
        check(lib.rq_mlp_create(n_in, h1, h2, n_out, seed, C.byref(h)))
        self._h = h
        n = C.c_int64()
        check(lib.rq_mlp_num_params(self._h, C.byref(n)))
        self.nparam = n.value

    def get_params(self) -> np.ndarray:
        p = np.empty(self.nparam, dtype=np.float32)
        check(lib.rq_mlp_get_params(self._h, _fp(p)))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparam
        check(lib.rq_mlp_set_params(self._h, _fp(p)))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty((x.shape[0], self.dims[3]), dtype=np.float32)
        check(lib.rq_mlp_forward(self._h, _fp(x), x.shape[0], _fp(y)))
        return y

    def gradients(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.empty(self.nparam, dtype=np.float32)
        loss = C.c_float()
        check(lib.rq_mlp_gradients(self._h, _fp(x), _fp(t), x.shape[0], C.byref(loss), _fp(g)))
        return loss.value, g

    def train(self, x, t, batch: int = 256, steps: int = 100, lr: float = 1e-3) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        check(lib.rq_mlp_train(self._h, _fp(x), _fp(t), x.shape[0], batch, steps, lr, C.byref(loss)))
        return loss.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            lib.rq_mlp_destroy(h)
            self._h = None


def linear_ramp(p: int, delta: float = 0.75):
    """Plain start: gamma_l = (l - 1/2)/p * delta, beta_l = (1 - (l - 1/2)/p) * delta, l = 1..p."""
    f = (np.arange(1, p + 1) - 0.5) / p
    return f * delta, (1.0 - f) * delta


def features(graphs) -> np.ndarray:
    return np.stack([graph_features(n, e) for n, e in graphs]).astype(np.float32)
