"""CPU oracle for the ruqu-core state-vector path -- TEST INFRASTRUCTURE ONLY.

Python (ctypes) view of ``oracle/liboracle.so``, the C++ restatement of the
reference's scalar engine (crates/ruqu-core/src/state.rs, gate.rs,
simulator.rs, mixed_precision.rs; crates/ruqu-algorithms/src/qaoa.rs, vqe.rs).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference legs may use it, and only as the checker / the timed CPU
baseline.  The product package ``ruqu_b200`` never imports it.

Parity status: gate matrices, gate kernels, measurement/collapse,
expectations, normalisation, fidelity and the QAOA/VQE drivers are pinned
against the reference's known-answer tests (tests/test_oracle_kats.py).  The
reference's RNG draws (rand 0.8.6 StdRng / ChaCha12) are not pinned by any
reference test and are replaced by the documented Philox4x32-10 stream, so
agreement with the Rust binary's concrete random draws is parity unpinned.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")

RQ_F32, RQ_F64 = 0, 1


class Gate(C.Structure):
    """Same layout as ``rq_gate`` in include/ruqu_cuda.h."""

    _fields_ = [("kind", C.c_int32), ("q0", C.c_uint32), ("q1", C.c_uint32), ("pad", C.c_uint32),
                ("angle", C.c_double), ("m", C.c_double * 8)]


class Measurement(C.Structure):
    _fields_ = [("qubit", C.c_uint32), ("result", C.c_int32), ("probability", C.c_double)]


class PauliOp(C.Structure):
    _fields_ = [("qubit", C.c_uint32), ("op", C.c_int32)]


def build() -> str:
    """Compile liboracle.so with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def _load() -> C.CDLL:
    if not os.path.exists(_SO):
        build()
    lib = C.CDLL(_SO)
    u32, u64, i32, dbl, vp = C.c_uint32, C.c_uint64, C.c_int32, C.c_double, C.c_void_p
    P = C.POINTER
    sig = {
        "orc_last_error": (C.c_char_p, []),
        "orc_philox": (None, [P(u32), P(u32), P(u32)]),
        "orc_uniform": (dbl, [u64, u32, u64]),
        "orc_state_new": (i32, [u32, i32, u64, i32, P(vp)]),
        "orc_state_from_amplitudes": (i32, [P(dbl), u64, u32, i32, u64, P(vp)]),
        "orc_state_free": (None, [vp]),
        "orc_apply": (i32, [vp, P(Gate), u64, P(Measurement), u64, P(u64), i32]),
        "orc_apply_noisy": (i32, [vp, P(Gate), u64, P(C.c_double), P(Measurement), u64, P(u64)]),
        "orc_apply_1q_matrix": (i32, [vp, u32, P(dbl)]),
        "orc_apply_2q_matrix": (i32, [vp, u32, u32, P(dbl)]),
        "orc_apply_kraus": (i32, [vp, u32, P(dbl), u32, P(i32), P(dbl)]),
        "orc_measure": (i32, [vp, u32, P(Measurement)]),
        "orc_reset_qubit": (i32, [vp, u32]),
        "orc_probabilities": (None, [vp, P(dbl)]),
        "orc_prob_qubit": (dbl, [vp, u32]),
        "orc_expectation": (dbl, [vp, P(PauliOp), u32]),
        "orc_expectation_hamiltonian": (dbl, [vp, P(dbl), P(PauliOp), P(u32), u32]),
        "orc_normalize": (None, [vp]),
        "orc_fidelity": (dbl, [vp, vp]),
        "orc_download": (None, [vp, P(dbl)]),
        "orc_upload": (None, [vp, P(dbl)]),
        "orc_draws": (u64, [vp]),
        "orc_run_shots_literal": (i32, [u32, i32, P(Gate), u64, u64, u64, P(u64)]),
        "orc_tree_sample": (None, [P(dbl), u32, P(u32), u32, u64, u64, P(u64)]),
        "orc_qaoa_cost": (dbl, [u32, P(u32), P(u32), P(dbl), u32, P(dbl), P(dbl), u32, i32]),
        "orc_qaoa_probabilities": (None, [u32, P(u32), P(u32), P(dbl), u32, P(dbl), P(dbl), u32, i32, P(dbl)]),
        "orc_run_qaoa": (i32, [u32, P(u32), P(u32), P(dbl), u32, u32, u32, dbl,
                               P(dbl), P(dbl), P(dbl), P(u32), P(dbl), P(u64), P(i32)]),
        "orc_circuit_energy": (dbl, [u32, i32, P(Gate), u64, P(dbl), P(PauliOp), P(u32), u32]),
        "orc_run_vqe": (i32, [u32, u32, P(dbl), P(PauliOp), P(u32), u32, u32, dbl, dbl,
                              P(dbl), P(dbl), P(u32), P(dbl), P(i32)]),
        "orc_num_threads": (i32, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _u32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _u64p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


class OracleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _check(rc: int):
    if rc != 0:
        raise OracleError(rc, lib().orc_last_error().decode())


# ---------------------------------------------------------------------------
# gate-list helpers: a gate list is a sequence of tuples
#   (kind, q0, q1, angle)  or  (kind, q0, q1, angle, m8)
# with kind codes of include/ruqu_cuda.h.
# ---------------------------------------------------------------------------

def gate_array(gates) -> C.Array:
    arr = (Gate * max(1, len(gates)))()
    for k, g in enumerate(gates):
        arr[k].kind = int(g[0])
        arr[k].q0 = int(g[1])
        arr[k].q1 = int(g[2]) if len(g) > 2 else 0
        arr[k].angle = float(g[3]) if len(g) > 3 else 0.0
        if len(g) > 4 and g[4] is not None:
            for i in range(8):
                arr[k].m[i] = float(g[4][i])
    return arr


def pauli_arrays(terms):
    """terms: list of Pauli strings, each a list of (qubit, op)."""
    offsets = np.zeros(len(terms) + 1, dtype=np.uint32)
    flat = []
    for k, t in enumerate(terms):
        flat.extend(t)
        offsets[k + 1] = len(flat)
    ops = (PauliOp * max(1, len(flat)))()
    for k, (q, o) in enumerate(flat):
        ops[k].qubit = int(q)
        ops[k].op = int(o)
    return ops, offsets


class OracleState:
    """Reference-semantics state (QuantumState / QuantumStateF32)."""

    def __init__(self, num_qubits: int, precision: int = RQ_F64, seed: int | None = 0, _handle=None):
        self.num_qubits = num_qubits
        self.precision = precision
        if _handle is not None:
            self._h = _handle
            return
        h = C.c_void_p()
        _check(lib().orc_state_new(num_qubits, precision, 0 if seed is None else seed,
                                   0 if seed is None else 1, C.byref(h)))
        self._h = h

    @classmethod
    def from_amplitudes(cls, amps: np.ndarray, num_qubits: int, precision: int = RQ_F64, seed: int = 0):
        a = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128)).view(np.float64)
        h = C.c_void_p()
        _check(lib().orc_state_from_amplitudes(_dp(a), len(a) // 2, num_qubits, precision, seed, C.byref(h)))
        return cls(num_qubits, precision, _handle=h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.orc_state_free(h)
            self._h = None

    def apply(self, gates, parallel: bool = False):
        arr = gate_array(gates)
        out = (Measurement * (len(gates) + 1))()
        nout = C.c_uint64()
        _check(lib().orc_apply(self._h, arr, len(gates), out, len(gates) + 1, C.byref(nout), 1 if parallel else 0))
        return [(out[k].qubit, bool(out[k].result), out[k].probability) for k in range(nout.value)]

    def apply_noisy(self, gates, rates):
        """run_with_config's gate loop with NoiseModel rates (depolarizing, bit_flip, phase_flip)."""
        arr = gate_array(gates)
        r = np.ascontiguousarray(rates, dtype=np.float64)
        out = (Measurement * (len(gates) + 1))()
        nout = C.c_uint64()
        _check(lib().orc_apply_noisy(self._h, arr, len(gates), _dp(r), out, len(gates) + 1, C.byref(nout)))
        return [(out[k].qubit, bool(out[k].result), out[k].probability) for k in range(nout.value)]

    def apply_1q_matrix(self, q, m8):
        m = np.ascontiguousarray(m8, dtype=np.float64)
        _check(lib().orc_apply_1q_matrix(self._h, q, _dp(m)))

    def apply_kraus(self, q, ops):
        """One trajectory step of a single-qubit channel (ops: k x 2 x 2 complex); (k, p)."""
        k = np.ascontiguousarray(np.asarray(ops, dtype=np.complex128).reshape(-1, 2, 2)).view(np.float64)
        k = np.ascontiguousarray(k.reshape(-1))
        chosen, prob = C.c_int32(), C.c_double()
        _check(lib().orc_apply_kraus(self._h, q, _dp(k), len(k) // 8, C.byref(chosen), C.byref(prob)))
        return chosen.value, prob.value

    def apply_2q_matrix(self, q1, q2, m32):
        m = np.ascontiguousarray(m32, dtype=np.float64)
        _check(lib().orc_apply_2q_matrix(self._h, q1, q2, _dp(m)))

    def measure(self, q):
        m = Measurement()
        _check(lib().orc_measure(self._h, q, C.byref(m)))
        return (m.qubit, bool(m.result), m.probability)

    def reset_qubit(self, q):
        _check(lib().orc_reset_qubit(self._h, q))

    def probabilities(self) -> np.ndarray:
        out = np.empty(1 << self.num_qubits, dtype=np.float64)
        lib().orc_probabilities(self._h, _dp(out))
        return out

    def probability_of_qubit(self, q) -> float:
        return lib().orc_prob_qubit(self._h, q)

    def expectation(self, ops) -> float:
        arr, _ = pauli_arrays([ops])
        return lib().orc_expectation(self._h, arr, len(ops))

    def expectation_hamiltonian(self, coeffs, terms) -> float:
        ops, off = pauli_arrays(terms)
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        return lib().orc_expectation_hamiltonian(self._h, _dp(c), ops, _u32p(off), len(terms))

    def normalize(self):
        lib().orc_normalize(self._h)

    def fidelity(self, other: "OracleState") -> float:
        return lib().orc_fidelity(self._h, other._h)

    def amplitudes(self) -> np.ndarray:
        out = np.empty(2 << self.num_qubits, dtype=np.float64)
        lib().orc_download(self._h, _dp(out))
        return out.view(np.complex128)

    def upload(self, amps: np.ndarray):
        a = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128)).view(np.float64)
        lib().orc_upload(self._h, _dp(a))


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.empty(4, dtype=np.uint32)
    lib().orc_philox(_u32p(c), _u32p(k), _u32p(out))
    return out


def uniform(seed: int, stream: int, index: int) -> float:
    return lib().orc_uniform(seed, stream, index)


def run_shots_literal(num_qubits, gates, shots, base_seed=42, precision=RQ_F64) -> np.ndarray:
    arr = gate_array(gates)
    out = np.empty(shots, dtype=np.uint64)
    _check(lib().orc_run_shots_literal(num_qubits, precision, arr, len(gates), shots, base_seed, _u64p(out)))
    return out


def tree_sample(probs: np.ndarray, num_qubits: int, qubits, base_seed: int, shots: int) -> np.ndarray:
    p = np.ascontiguousarray(probs, dtype=np.float64)
    q = np.ascontiguousarray(qubits, dtype=np.uint32)
    out = np.empty(shots, dtype=np.uint64)
    lib().orc_tree_sample(_dp(p), num_qubits, _u32p(q), len(q), base_seed, shots, _u64p(out))
    return out


def _edges(graph_edges):
    e = np.asarray(graph_edges, dtype=np.float64).reshape(-1, 3)
    ei = np.ascontiguousarray(e[:, 0].astype(np.uint32))
    ej = np.ascontiguousarray(e[:, 1].astype(np.uint32))
    w = np.ascontiguousarray(e[:, 2])
    return ei, ej, w


def qaoa_cost(n, edges, gammas, betas, precision=RQ_F64) -> float:
    ei, ej, w = _edges(edges)
    g = np.ascontiguousarray(gammas, dtype=np.float64)
    b = np.ascontiguousarray(betas, dtype=np.float64)
    return lib().orc_qaoa_cost(n, _u32p(ei), _u32p(ej), _dp(w), len(w), _dp(g), _dp(b), len(g), precision)


def qaoa_probabilities(n, edges, gammas, betas, precision=RQ_F64) -> np.ndarray:
    ei, ej, w = _edges(edges)
    g = np.ascontiguousarray(gammas, dtype=np.float64)
    b = np.ascontiguousarray(betas, dtype=np.float64)
    out = np.empty(1 << n, dtype=np.float64)
    lib().orc_qaoa_probabilities(n, _u32p(ei), _u32p(ej), _dp(w), len(w), _dp(g), _dp(b), len(g), precision, _dp(out))
    return out


def run_qaoa(n, edges, p, max_iterations, learning_rate):
    ei, ej, w = _edges(edges)
    g = np.empty(p)
    b = np.empty(p)
    hist = np.empty(max(1, max_iterations))
    iters = C.c_uint32()
    best = C.c_double()
    bits = C.c_uint64()
    conv = C.c_int32()
    _check(lib().orc_run_qaoa(n, _u32p(ei), _u32p(ej), _dp(w), len(w), p, max_iterations, learning_rate,
                              _dp(g), _dp(b), _dp(hist), C.byref(iters), C.byref(best), C.byref(bits), C.byref(conv)))
    return dict(gammas=g, betas=b, history=hist[:iters.value].copy(), best_cut_value=best.value,
                best_bits=bits.value, converged=bool(conv.value))


def circuit_energy(n, gates, coeffs, terms, precision=RQ_F64) -> float:
    arr = gate_array(gates)
    ops, off = pauli_arrays(terms)
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    return lib().orc_circuit_energy(n, precision, arr, len(gates), _dp(c), ops, _u32p(off), len(terms))


def run_vqe(n, depth, coeffs, terms, max_iterations, threshold, learning_rate):
    ops, off = pauli_arrays(terms)
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    npar = 2 * n * depth
    bp = np.empty(npar)
    hist = np.empty(max(1, max_iterations))
    iters = C.c_uint32()
    best = C.c_double()
    conv = C.c_int32()
    _check(lib().orc_run_vqe(n, depth, _dp(c), ops, _u32p(off), len(terms), max_iterations, threshold, learning_rate,
                             _dp(bp), _dp(hist), C.byref(iters), C.byref(best), C.byref(conv)))
    return dict(best_params=bp, history=hist[:iters.value].copy(), best_energy=best.value,
                converged=bool(conv.value))


def num_threads() -> int:
    return lib().orc_num_threads()
