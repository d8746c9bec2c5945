"""Batched QAOA-MaxCut on the GPU (rq_qaoa_batch_* of include/ruqu_cuda.h).

Evaluates the circuit of build_qaoa_circuit (crates/ruqu-algorithms/src/qaoa.rs:125-153)
for many graphs and many (gamma, beta) sets in one call, returning the expected cut of
evaluate_qaoa_cost (qaoa.rs:179-201) per circuit and, optionally, the best cut among
shots drawn with run_shots semantics (crates/ruqu-core/src/simulator.rs:107-147).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import RQ_F32, RQ_F64, lib
from .error import check


def _u32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class QaoaBatch:
    """graphs: sequence of (num_nodes, [(u, v), ...]) simple unweighted graphs."""

    def __init__(self, graphs, p: int, precision: str = "f32"):
        self.graphs = [(int(n), [(int(u), int(v)) for u, v in e]) for n, e in graphs]
        self.p = int(p)
        self.precision = precision
        nodes = np.ascontiguousarray([g[0] for g in self.graphs], dtype=np.uint32)
        offs = np.zeros(len(self.graphs) + 1, dtype=np.uint32)
        flat = []
        for k, (_, e) in enumerate(self.graphs):
            for u, v in e:
                flat += [u, v]
            offs[k + 1] = offs[k] + len(e)
        edges = np.ascontiguousarray(flat if flat else [0, 0], dtype=np.uint32)
        h = C.c_void_p()
        check(lib.rq_qaoa_batch_create(len(self.graphs), _u32p(nodes), _u32p(offs), _u32p(edges), self.p,
                                       RQ_F32 if precision == "f32" else RQ_F64, C.byref(h)))
        self._h = h
        self.nsets = 1

    def run(self, gammas, betas, shots: int = 0, seed: int = 0):
        """gammas, betas: (ninst, p) or (ninst, nsets, p).  Returns energies of shape
        (ninst,) or (ninst, nsets), plus best_bits / best_cut when shots > 0."""
        g = np.asarray(gammas, dtype=np.float64)
        b = np.asarray(betas, dtype=np.float64)
        squeeze = g.ndim == 2
        if squeeze:
            g = g[:, None, :]
            b = b[:, None, :]
        ninst, nsets, p = g.shape
        assert ninst == len(self.graphs) and p == self.p and b.shape == g.shape
        g = np.ascontiguousarray(g.reshape(-1))
        b = np.ascontiguousarray(b.reshape(-1))
        e = np.empty(ninst * nsets)
        bb = np.zeros(ninst * nsets, dtype=np.uint64)
        bc = np.zeros(ninst * nsets, dtype=np.uint32)
        check(lib.rq_qaoa_batch_run(self._h, nsets, _dp(g), _dp(b), _dp(e), int(shots), int(seed) & (2**64 - 1),
                                    bb.ctypes.data_as(C.POINTER(C.c_uint64)), _u32p(bc)))
        self.nsets = nsets
        shape = (ninst,) if squeeze else (ninst, nsets)
        out = {"energies": e.reshape(shape)}
        if shots:
            out["best_bits"] = bb.reshape(shape)
            out["best_cut"] = bc.reshape(shape)
        return out

    def gradient(self, gammas, betas):
        """Energies and exact gradients (ninst x 2p: d/dgamma_1..p, then d/dbeta_1..p) of one
        circuit per graph, by the adjoint pass on the GPU."""
        g = np.ascontiguousarray(np.array(gammas, dtype=np.float64).reshape(len(self.graphs), self.p))
        b = np.ascontiguousarray(np.array(betas, dtype=np.float64).reshape(len(self.graphs), self.p))
        e = np.empty(len(self.graphs))
        grad = np.empty((len(self.graphs), 2 * self.p))
        check(lib.rq_qaoa_batch_gradient(self._h, _dp(g), _dp(b), _dp(e), _dp(grad)))
        self.nsets = 1
        return e, grad

    def optimize(self, gammas, betas, steps: int, lr: float = 0.05, target=None, rtol: float = 1e-5,
                 gradient: str = "adjoint"):
        """Adam on the GPU.  gradient = "adjoint" (exact gradients) or "shift" (the rule of
        run_qaoa, qaoa.rs:275-297, zero up to rounding for unit edge weights).
        Returns (gammas, betas, energies, steps_taken)."""
        mode = {"adjoint": _capi.RQ_QAOA_GRAD_ADJOINT, "shift": _capi.RQ_QAOA_GRAD_SHIFT}[gradient]
        g = np.ascontiguousarray(np.array(gammas, dtype=np.float64).reshape(len(self.graphs), self.p))
        b = np.ascontiguousarray(np.array(betas, dtype=np.float64).reshape(len(self.graphs), self.p))
        e = np.empty(len(self.graphs))
        st = np.empty(len(self.graphs), dtype=np.uint32)
        tp = None
        if target is not None:
            t = np.ascontiguousarray(target, dtype=np.float64)
            tp = _dp(t)
        check(lib.rq_qaoa_batch_optimize(self._h, int(steps), float(lr), _dp(g), _dp(b), tp, float(rtol), mode,
                                         _dp(e), _u32p(st)))
        self.nsets = 1 if gradient == "adjoint" else 1 + 4 * self.p
        return g, b, e, st

    def optimize_precond(self, gammas, betas, precond, steps: int, alpha: float = 0.8, target=None,
                         rtol: float = 1e-5):
        """Preconditioned ascent with exact gradients: theta += alpha_i P_i grad E per instance
        (precond: ninst x 2p x 2p; alpha_i halves when an instance's energy falls).
        Returns (gammas, betas, energies, steps_taken)."""
        g = np.ascontiguousarray(np.array(gammas, dtype=np.float64).reshape(len(self.graphs), self.p))
        b = np.ascontiguousarray(np.array(betas, dtype=np.float64).reshape(len(self.graphs), self.p))
        P = np.ascontiguousarray(np.asarray(precond, dtype=np.float64).reshape(len(self.graphs), 2 * self.p,
                                                                                 2 * self.p))
        e = np.empty(len(self.graphs))
        st = np.empty(len(self.graphs), dtype=np.uint32)
        tp = None
        if target is not None:
            t = np.ascontiguousarray(target, dtype=np.float64)
            tp = _dp(t)
        check(lib.rq_qaoa_batch_optimize_precond(self._h, int(steps), _dp(P), float(alpha), _dp(g), _dp(b), tp,
                                                 float(rtol), _dp(e), _u32p(st)))
        self.nsets = 1
        return g, b, e, st

    def set_convergence(self, tol: float) -> None:
        """run_qaoa's convergence rule (qaoa.rs:266-269) for optimize / optimize_precond: an
        instance stops once its energy changed by less than tol in a step (0 turns it off)."""
        check(lib.rq_qaoa_batch_set_convergence(self._h, float(tol)))

    def state(self, circuit: int) -> np.ndarray:
        n = self.graphs[circuit // self.nsets][0]
        out = np.empty(2 << n)
        check(lib.rq_qaoa_batch_state(self._h, int(circuit), _dp(out)))
        return out.view(np.complex128)

    def last_ms(self) -> float:
        ms = C.c_float()
        check(lib.rq_qaoa_batch_last_ms(self._h, C.byref(ms)))
        return ms.value

    def last_profile(self) -> dict:
        """Device time and algorithmic work of the last run / gradient, by kernel kind."""
        out = np.zeros(6)
        check(lib.rq_qaoa_batch_last_profile(self._h, _dp(out)))
        return {"sweep_bytes": out[0], "sweep_ms": out[1], "sample_bytes": out[2], "sample_ms": out[3],
                "adjoint_bytes": out[4], "adjoint_ms": out[5]}

    def set_state_budget(self, nbytes: int) -> None:
        check(lib.rq_qaoa_batch_set_state_budget(self._h, int(nbytes)))

    def set_graphs(self, enable: bool) -> None:
        """Capture repeated runs of one shape as a CUDA graph (default on)."""
        check(lib.rq_qaoa_batch_set_graphs(self._h, 1 if enable else 0))

    def last_graph(self) -> dict:
        """Whether the last run / gradient launched its captured graph, and its kernel count."""
        r, k = C.c_int32(), C.c_uint64()
        check(lib.rq_qaoa_batch_last_graph(self._h, C.byref(r), C.byref(k)))
        return {"replayed": bool(r.value), "kernels": int(k.value)}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            lib.rq_qaoa_batch_destroy(h)
            self._h = None


class VqeBatch:
    """Batched VQE energies / parameter-shift gradients (rq_vqe_batch_* of include/ruqu_cuda.h).

    Ansatz: per layer Ry(theta) on every qubit then CZ(q, q+1) (parameters layer-major);
    Hamiltonian: coeffs[k] * P_k with P_k a list of (qubit, PauliOp)."""

    def __init__(self, num_qubits: int, depth: int, coeffs, strings, precision: str = "f32"):
        from .state import pauli_array
        self.n, self.depth = int(num_qubits), int(depth)
        self.P = self.n * self.depth
        ops, off = pauli_array(strings)
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        h = C.c_void_p()
        check(lib.rq_vqe_batch_create(self.n, self.depth, _dp(c), ops, _u32p(off), len(strings),
                                      RQ_F32 if precision == "f32" else RQ_F64, C.byref(h)))
        self._h = h

    def run(self, params, gradient=False):
        """params: (nsets, P).  Returns energies (nsets,) and, with a gradient, (nsets, P)
        gradients: gradient=True or "shift" for the parameter-shift rule of run_vqe
        (vqe.rs:186-198, 1 + 2P circuits per set), "adjoint" for the same derivative by one
        backward pass per set."""
        mode = {False: _capi.RQ_VQE_GRAD_NONE, None: _capi.RQ_VQE_GRAD_NONE, True: _capi.RQ_VQE_GRAD_SHIFT,
                "shift": _capi.RQ_VQE_GRAD_SHIFT, "adjoint": _capi.RQ_VQE_GRAD_ADJOINT}[gradient]
        p = np.ascontiguousarray(np.atleast_2d(np.asarray(params, dtype=np.float64)))
        nsets = p.shape[0]
        if p.shape[1] != self.P:
            raise ValueError(f"params must have {self.P} columns")
        e = np.empty(nsets)
        g = np.empty((nsets, self.P)) if mode else np.empty(1)
        check(lib.rq_vqe_batch_run(self._h, nsets, _dp(p), mode, _dp(e), _dp(g)))
        return (e, g) if mode else e

    def last_profile(self) -> dict:
        """Device time and algorithmic work of the last run, by kernel kind."""
        out = np.zeros(6)
        check(lib.rq_vqe_batch_last_profile(self._h, _dp(out)))
        return {"sweep_bytes": out[0], "sweep_ms": out[1], "energy_flops": out[2], "energy_ms": out[3],
                "adjoint_bytes": out[4], "adjoint_ms": out[5]}

    def last_ms(self) -> float:
        ms = C.c_float()
        check(lib.rq_vqe_batch_last_ms(self._h, C.byref(ms)))
        return ms.value

    def set_graphs(self, enable: bool) -> None:
        """Capture repeated runs of one shape as a CUDA graph (default on)."""
        check(lib.rq_vqe_batch_set_graphs(self._h, 1 if enable else 0))

    def last_graph(self) -> dict:
        """Whether the last run launched its captured graph, and its kernel count."""
        r, k = C.c_int32(), C.c_uint64()
        check(lib.rq_vqe_batch_last_graph(self._h, C.byref(r), C.byref(k)))
        return {"replayed": bool(r.value), "kernels": int(k.value)}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            lib.rq_vqe_batch_destroy(h)
            self._h = None
