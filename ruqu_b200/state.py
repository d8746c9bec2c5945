"""Device-resident state vector (crates/ruqu-core/src/state.rs:18-450).

``QuantumState`` keeps its 2^n amplitudes in HBM (interleaved complex f64,
or f32 like ``QuantumStateF32``, mixed_precision.rs:193-549) and forwards
every method to libruqu_cuda.so.  Host copies exist only when the caller asks
for them (``state_vector``, ``probabilities``, ``amplitudes_mut``).
"""
from __future__ import annotations

import contextlib
import ctypes as C

import numpy as np

from . import _capi
from ._capi import RQ_F32, RQ_F64, RqMeasurement, RqPauliOp, RqPlanStats, lib
from .circuit import gates_to_array
from .error import check
from .gate import Gate
from .types import Hamiltonian, MeasurementOutcome, PauliString

MAX_QUBITS = 32        # state.rs:15
MAX_QUBITS_F32 = 33    # mixed_precision.rs:185


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _precision(p) -> int:
    if p in (RQ_F64, "f64", "float64", np.float64, np.complex128, None):
        return RQ_F64
    if p in (RQ_F32, "f32", "float32", np.float32, np.complex64):
        return RQ_F32
    raise ValueError(f"unknown precision {p!r}")


def pauli_array(strings):
    """Flatten Pauli strings into (rq_pauli_op array, offsets)."""
    offsets = np.zeros(len(strings) + 1, dtype=np.uint32)
    flat = []
    for k, ps in enumerate(strings):
        ops = ps.ops if isinstance(ps, PauliString) else ps
        flat.extend(ops)
        offsets[k + 1] = len(flat)
    arr = (RqPauliOp * max(1, len(flat)))()
    for k, (q, o) in enumerate(flat):
        arr[k].qubit = int(q)
        arr[k].op = int(o)
    return arr, offsets


class QuantumState:
    """|psi> on the GPU.  Construct with ``QuantumState(n)``, ``new_with_seed`` or ``from_amplitudes``."""

    def __init__(self, num_qubits: int, seed: int | None = None, precision="f64", _handle=None):
        self._prec = _precision(precision)
        self._record: list = []
        if _handle is not None:
            self._h = _handle
        else:
            h = C.c_void_p()
            check(lib.rq_state_create(int(num_qubits), self._prec, 0 if seed is None else int(seed) & (2**64 - 1),
                                      0 if seed is None else 1, C.byref(h)))
            self._h = h
        n = C.c_uint32()
        check(lib.rq_state_num_qubits(self._h, C.byref(n)))
        self._n = n.value

    # ---- constructors (state.rs:31-96) ----
    @classmethod
    def new(cls, num_qubits: int, precision="f64") -> "QuantumState":
        return cls(num_qubits, None, precision)

    @classmethod
    def new_with_seed(cls, num_qubits: int, seed: int, precision="f64") -> "QuantumState":
        return cls(num_qubits, seed, precision)

    @classmethod
    def from_amplitudes(cls, amps, num_qubits: int, precision="f64", seed: int = 0) -> "QuantumState":
        a = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128)).view(np.float64)
        h = C.c_void_p()
        check(lib.rq_state_from_amplitudes(_dp(a), len(a) // 2, int(num_qubits), _precision(precision),
                                           int(seed), C.byref(h)))
        return cls(num_qubits, precision=precision, _handle=h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            lib.rq_state_destroy(h)
            self._h = None

    # ---- accessors (state.rs:102-154) ----
    def num_qubits(self) -> int:
        return self._n

    def num_amplitudes(self) -> int:
        return 1 << self._n

    @property
    def precision(self) -> str:
        return "f32" if self._prec == RQ_F32 else "f64"

    @property
    def handle(self):
        return self._h

    def state_vector(self) -> np.ndarray:
        out = np.empty(2 << self._n, dtype=np.float64)
        check(lib.rq_state_download(self._h, _dp(out)))
        return out.view(np.complex128)

    @contextlib.contextmanager
    def amplitudes_mut(self):
        """Host-editable copy written back on exit (state.rs:118-124 returns a slice instead)."""
        a = self.state_vector()
        yield a
        self.set_amplitudes(a)

    def set_amplitudes(self, amps) -> None:
        a = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128)).view(np.float64)
        if a.size != 2 << self._n:
            raise ValueError("amplitude count does not match 2^num_qubits")
        check(lib.rq_state_upload(self._h, _dp(a)))

    def probabilities(self) -> np.ndarray:
        out = np.empty(1 << self._n, dtype=np.float64)
        check(lib.rq_state_probabilities(self._h, _dp(out)))
        return out

    def probability_of_qubit(self, qubit: int) -> float:
        out = C.c_double()
        check(lib.rq_state_probability_of_qubit(self._h, int(qubit), C.byref(out)))
        return out.value

    def measurement_record(self) -> list:
        return list(self._record)

    @staticmethod
    def estimate_memory(num_qubits: int, precision="f64") -> int:
        return (1 << num_qubits) * (8 if _precision(precision) == RQ_F32 else 16)

    def device_pointer(self):
        """(device pointer of the amplitudes, CUDA stream handle) for zero-copy interop."""
        p, s = C.c_void_p(), C.c_void_p()
        check(lib.rq_state_device_ptr(self._h, C.byref(p), C.byref(s)))
        return p.value, s.value

    def synchronize(self) -> None:
        check(lib.rq_state_synchronize(self._h))

    def reset(self) -> None:
        """Back to |0...0> with the measurement stream rewound."""
        check(lib.rq_state_reset(self._h))
        self._record.clear()

    # ---- gates (state.rs:158-276) ----
    def apply_gate(self, gate: Gate) -> list:
        return self.apply_gates([gate])

    def apply_gates(self, gates, mode: int = _capi.RQ_EXEC_AUTO) -> list:
        arr = gates if isinstance(gates, C.Array) else gates_to_array(gates)
        n = len(gates)
        out = (RqMeasurement * max(1, n))()
        nout = C.c_uint64()
        check(lib.rq_state_apply_mode(self._h, arr, n, int(mode), out, n, C.byref(nout)))
        res = [MeasurementOutcome(out[k].qubit, bool(out[k].result), out[k].probability) for k in range(nout.value)]
        self._record.extend(res)
        return res

    def apply_gates_noisy(self, gates, noise) -> list:
        """The gates with per-gate Pauli noise drawn from this state's stream, as
        Simulator::run_with_config applies a NoiseModel (simulator.rs:67-78, 177-221)."""
        arr = gates if isinstance(gates, C.Array) else gates_to_array(gates)
        n = len(gates)
        nm = _capi.RqNoiseModel(float(noise.depolarizing_rate), float(noise.bit_flip_rate),
                                float(noise.phase_flip_rate))
        out = (RqMeasurement * max(1, n))()
        nout = C.c_uint64()
        check(lib.rq_state_apply_noisy(self._h, arr, n, C.byref(nm), out, n, C.byref(nout)))
        res = [MeasurementOutcome(out[k].qubit, bool(out[k].result), out[k].probability) for k in range(nout.value)]
        self._record.extend(res)
        return res

    def negate_amplitudes(self, indices) -> None:
        """amps[i] = -amps[i] for every listed index, on the device (the oracle step that
        run_grover does through amplitudes_mut, grover.rs:128-139)."""
        idx = np.ascontiguousarray(np.asarray(indices, dtype=np.uint64).reshape(-1))
        check(lib.rq_state_negate_amplitudes(self._h, idx.ctypes.data_as(C.POINTER(C.c_uint64)), idx.size))

    def half_copy(self, qubit: int, value: int, device_ptr: int, unpack: bool = False) -> None:
        """Copy the amplitudes whose bit `qubit` equals `value` (in the order of the other
        bits) to the device buffer at device_ptr, or back from it (unpack=True): the
        exchange step of a distributed state.  Runs on this state's stream."""
        check(lib.rq_state_half_copy(self._h, int(qubit), int(value), C.c_void_p(int(device_ptr)),
                                     _capi.RQ_HALF_UNPACK if unpack else _capi.RQ_HALF_PACK))

    def negate_all_except(self, keep: int = 0) -> None:
        """amps[i] = -amps[i] for every i != keep, on the device (grover.rs:144-153)."""
        check(lib.rq_state_negate_all_except(self._h, int(keep)))

    def apply_single_qubit_gate(self, qubit: int, matrix) -> None:
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128).reshape(2, 2)).view(np.float64)
        check(lib.rq_state_apply_1q_matrix(self._h, int(qubit), _dp(m)))

    def apply_two_qubit_gate(self, q1: int, q2: int, matrix) -> None:
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128).reshape(4, 4)).view(np.float64)
        check(lib.rq_state_apply_2q_matrix(self._h, int(q1), int(q2), _dp(m)))

    def apply_kraus(self, qubit: int, ops) -> tuple[int, float]:
        """One quantum-trajectory step of the single-qubit channel with Kraus operators
        ``ops`` (k x 2 x 2 complex, e.g. from ``ruqu_b200.noise``): operator k is picked
        with probability tr(K_k rho K_k^dagger) by the next draw of this state's stream
        and applied renormalised.  Returns (k, its probability)."""
        k = np.ascontiguousarray(np.asarray(ops, dtype=np.complex128).reshape(-1, 2, 2)).view(np.float64)
        chosen, prob = C.c_int32(), C.c_double()
        check(lib.rq_state_apply_kraus(self._h, int(qubit), _dp(k), k.size // 8, C.byref(chosen), C.byref(prob)))
        return chosen.value, prob.value

    # ---- measurement (state.rs:288-352) ----
    def measure(self, qubit: int) -> MeasurementOutcome:
        m = RqMeasurement()
        check(lib.rq_state_measure(self._h, int(qubit), C.byref(m)))
        o = MeasurementOutcome(m.qubit, bool(m.result), m.probability)
        self._record.append(o)
        return o

    def measure_all(self) -> list:
        out = (RqMeasurement * self._n)()
        check(lib.rq_state_measure_all(self._h, out))
        res = [MeasurementOutcome(out[k].qubit, bool(out[k].result), out[k].probability) for k in range(self._n)]
        self._record.extend(res)
        return res

    def reset_qubit(self, qubit: int) -> None:
        check(lib.rq_state_reset_qubit(self._h, int(qubit)))

    def sample(self, shots: int, base_seed: int = 42, qubits=None) -> np.ndarray:
        """Shot bitstrings (bit q = outcome of qubit q) reproducing Simulator::run_shots' draws."""
        qs = np.ascontiguousarray(range(self._n) if qubits is None else qubits, dtype=np.uint32)
        out = np.empty(int(shots), dtype=np.uint64)
        check(lib.rq_state_sample(self._h, qs.ctypes.data_as(C.POINTER(C.c_uint32)), len(qs),
                                  int(base_seed) & (2**64 - 1), int(shots),
                                  out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out

    def tree_build(self, qubits) -> None:
        """Build the FP64 prefix tree of the sampler over ``qubits`` (in that order, the
        rest after them) from the current amplitudes."""
        qs = np.ascontiguousarray(qubits, dtype=np.uint32)
        check(lib.rq_state_tree_build(self._h, qs.ctypes.data_as(C.POINTER(C.c_uint32)), len(qs)))

    def tree_lookup(self, level: int, index) -> np.ndarray:
        """Entries ``index`` of tree level ``level``: sums of |a|^2 over the amplitudes whose
        first ``level`` tree qubits take the bits of the index."""
        idx = np.ascontiguousarray(index, dtype=np.uint64)
        out = np.empty(len(idx), dtype=np.float64)
        check(lib.rq_state_tree_lookup(self._h, int(level), idx.ctypes.data_as(C.POINTER(C.c_uint64)), len(idx),
                                       _dp(out)))
        return out

    # ---- expectations (state.rs:362-408) ----
    def expectation_value(self, pauli) -> float:
        arr, off = pauli_array([pauli])
        out = C.c_double()
        check(lib.rq_state_expectation_value(self._h, arr, int(off[1]), C.byref(out)))
        return out.value

    def expectation_values(self, paulis) -> np.ndarray:
        """Many Pauli strings, one device call (strings sharing an X/Y pattern share one pass)."""
        arr, off = pauli_array(paulis)
        out = np.empty(len(paulis), dtype=np.float64)
        check(lib.rq_state_expectation_batch(self._h, arr, off.ctypes.data_as(C.POINTER(C.c_uint32)),
                                             len(paulis), _dp(out)))
        return out

    def expectation_hamiltonian(self, h: Hamiltonian) -> float:
        coeffs = np.ascontiguousarray([c for c, _ in h.terms], dtype=np.float64)
        arr, off = pauli_array([ps for _, ps in h.terms])
        out = C.c_double()
        check(lib.rq_state_expectation_hamiltonian(self._h, _dp(coeffs), arr,
                                                   off.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                   len(h.terms), C.byref(out)))
        return out.value

    # ---- normalisation & fidelity (state.rs:415-435) ----
    def norm_sq(self) -> float:
        out = C.c_double()
        check(lib.rq_state_norm_sq(self._h, C.byref(out)))
        return out.value

    def normalize(self) -> None:
        check(lib.rq_state_normalize(self._h))

    def fidelity(self, other: "QuantumState") -> float:
        out = C.c_double()
        check(lib.rq_state_fidelity(self._h, other._h, C.byref(out)))
        return out.value


class Plan:
    """A unitary gate list prepared once for states of one shape (rq_plan_create).

    ``execute(state)`` only launches kernels on the state's stream; the host
    planning and the upload of the gate tables happen here, once.
    """

    def __init__(self, state: QuantumState, gates, mode: int = _capi.RQ_EXEC_AUTO, local_qubits: int = 0):
        """local_qubits (tensor-core modes, complex f32): the sweep tile size, 12-13, or 12-14
        for RQ_EXEC_SWEEP_TC16 (rq_plan_create_tiled); 0 = the default."""
        arr = gates if isinstance(gates, C.Array) else gates_to_array(gates)
        h = C.c_void_p()
        if local_qubits:
            check(lib.rq_plan_create_tiled(state.handle, arr, len(gates), int(mode), int(local_qubits), C.byref(h)))
        else:
            check(lib.rq_plan_create(state.handle, arr, len(gates), int(mode), C.byref(h)))
        self._h = h

    def execute(self, state: QuantumState) -> None:
        check(lib.rq_plan_execute(state.handle, self._h))

    def update(self, state: QuantumState, gates) -> None:
        """New angles (or matrices) for the same gate kinds and qubits (rq_plan_update): the
        planning is kept, the matrix tables and operand images are rebuilt in stream order on
        the state's stream.  Raises CircuitError if the structure differs."""
        arr = gates if isinstance(gates, C.Array) else gates_to_array(gates)
        check(lib.rq_plan_update(state.handle, self._h, arr, len(gates)))

    def stats(self) -> dict:
        st = RqPlanStats()
        check(lib.rq_plan_get_stats(self._h, C.byref(st)))
        return {k: int(getattr(st, k)) for k, _ in RqPlanStats._fields_}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            lib.rq_plan_destroy(h)
            self._h = None


def set_device(device: int) -> None:
    """Device for states created afterwards on this thread."""
    check(lib.rq_device_set(int(device)))
