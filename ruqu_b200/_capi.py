"""ctypes binding of libruqu_cuda.so (the C ABI declared in include/ruqu_cuda.h).

The library is the only compute path: if it is missing this module raises
at import, and every call that fails on the device raises QuantumError.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libruqu_cuda.so")

RQ_F32, RQ_F64 = 0, 1
RQ_QAOA_GRAD_ADJOINT, RQ_QAOA_GRAD_SHIFT = 0, 1
RQ_VQE_GRAD_NONE, RQ_VQE_GRAD_SHIFT, RQ_VQE_GRAD_ADJOINT = 0, 1, 2
RQ_HALF_PACK, RQ_HALF_UNPACK = 0, 1
RQ_EXEC_AUTO, RQ_EXEC_PER_GATE, RQ_EXEC_SWEEP, RQ_EXEC_SWEEP_TC, RQ_EXEC_SWEEP_TC_FAST, RQ_EXEC_SWEEP_TC16 = range(6)

(RQ_OK, RQ_ERR_QUBIT_LIMIT_EXCEEDED, RQ_ERR_INVALID_QUBIT_INDEX, RQ_ERR_MEMORY_ALLOCATION,
 RQ_ERR_INVALID_STATE_VECTOR, RQ_ERR_CIRCUIT, RQ_ERR_CUDA, RQ_ERR_TIMEOUT, RQ_ERR_INVALID_ARGUMENT) = range(9)


class RqGate(C.Structure):
    _fields_ = [("kind", C.c_int32), ("q0", C.c_uint32), ("q1", C.c_uint32), ("pad", C.c_uint32),
                ("angle", C.c_double), ("m", C.c_double * 8)]


class RqMeasurement(C.Structure):
    _fields_ = [("qubit", C.c_uint32), ("result", C.c_int32), ("probability", C.c_double)]


class RqNoiseModel(C.Structure):
    _fields_ = [("depolarizing_rate", C.c_double), ("bit_flip_rate", C.c_double), ("phase_flip_rate", C.c_double)]


class RqPauliOp(C.Structure):
    _fields_ = [("qubit", C.c_uint32), ("op", C.c_int32)]


class RqPlanStats(C.Structure):
    _fields_ = [("gates", C.c_uint64), ("launches", C.c_uint64), ("sweeps", C.c_uint64), ("phases", C.c_uint64),
                ("ops", C.c_uint64), ("hbm_bytes", C.c_uint64), ("dense_ops", C.c_uint64),
                ("exec_mode", C.c_uint64), ("local_qubits", C.c_uint64)]


# name -> (restype, argtypes); every symbol here is declared in include/ruqu_cuda.h
_P = C.POINTER
_u32, _u64, _i32, _dbl, _vp = C.c_uint32, C.c_uint64, C.c_int32, C.c_double, C.c_void_p
SIGNATURES = {
    "rq_last_error_message": (C.c_char_p, []),
    "rq_version": (_i32, []),
    "rq_uniform": (_dbl, [_u64, _u32, _u64]),
    "rq_device_set": (C.c_int, [_i32]),
    "rq_device_count": (C.c_int, [_P(_i32)]),
    "rq_plan_create": (C.c_int, [_vp, _P(RqGate), _u64, _i32, _P(_vp)]),
    "rq_plan_create_tiled": (C.c_int, [_vp, C.c_void_p, _u64, _i32, _u32, _P(_vp)]),
    "rq_plan_execute": (C.c_int, [_vp, _vp]),
    "rq_plan_update": (C.c_int, [_vp, _vp, _P(RqGate), _u64]),
    "rq_plan_get_stats": (C.c_int, [_vp, _P(RqPlanStats)]),
    "rq_plan_destroy": (C.c_int, [_vp]),
    "rq_state_create": (C.c_int, [_u32, _i32, _u64, _i32, _P(_vp)]),
    "rq_state_from_amplitudes": (C.c_int, [_P(_dbl), _u64, _u32, _i32, _u64, _P(_vp)]),
    "rq_state_destroy": (C.c_int, [_vp]),
    "rq_state_reset": (C.c_int, [_vp]),
    "rq_state_num_qubits": (C.c_int, [_vp, _P(_u32)]),
    "rq_state_precision": (C.c_int, [_vp, _P(_i32)]),
    "rq_state_device_ptr": (C.c_int, [_vp, _P(_vp), _P(_vp)]),
    "rq_state_synchronize": (C.c_int, [_vp]),
    "rq_debug_set_wait_limit": (C.c_int, [_u32]),
    "rq_state_apply": (C.c_int, [_vp, _P(RqGate), _u64, _P(RqMeasurement), _u64, _P(_u64)]),
    "rq_state_apply_mode": (C.c_int, [_vp, _P(RqGate), _u64, _i32, _P(RqMeasurement), _u64, _P(_u64)]),
    "rq_state_apply_noisy": (C.c_int, [_vp, _P(RqGate), _u64, _P(RqNoiseModel), _P(RqMeasurement), _u64, _P(_u64)]),
    "rq_state_negate_amplitudes": (C.c_int, [_vp, _P(_u64), _u64]),
    "rq_state_negate_all_except": (C.c_int, [_vp, _u64]),
    "rq_state_half_copy": (C.c_int, [_vp, _u32, _u32, _vp, _i32]),
    "rq_state_apply_1q_matrix": (C.c_int, [_vp, _u32, _P(_dbl)]),
    "rq_state_apply_2q_matrix": (C.c_int, [_vp, _u32, _u32, _P(_dbl)]),
    "rq_state_measure": (C.c_int, [_vp, _u32, _P(RqMeasurement)]),
    "rq_state_apply_kraus": (C.c_int, [_vp, _u32, _P(_dbl), _u32, _P(_i32), _P(_dbl)]),
    "rq_state_measure_all": (C.c_int, [_vp, _P(RqMeasurement)]),
    "rq_state_reset_qubit": (C.c_int, [_vp, _u32]),
    "rq_state_sample": (C.c_int, [_vp, _P(_u32), _u32, _u64, _u64, _P(_u64)]),
    "rq_state_tree_build": (C.c_int, [_vp, _P(_u32), _u32]),
    "rq_state_tree_lookup": (C.c_int, [_vp, _u32, _P(_u64), _u64, _P(_dbl)]),
    "rq_state_probabilities": (C.c_int, [_vp, _P(_dbl)]),
    "rq_state_probability_of_qubit": (C.c_int, [_vp, _u32, _P(_dbl)]),
    "rq_state_expectation_value": (C.c_int, [_vp, _P(RqPauliOp), _u32, _P(_dbl)]),
    "rq_state_expectation_batch": (C.c_int, [_vp, _P(RqPauliOp), _P(_u32), _u32, _P(_dbl)]),
    "rq_state_expectation_hamiltonian": (C.c_int, [_vp, _P(_dbl), _P(RqPauliOp), _P(_u32), _u32, _P(_dbl)]),
    "rq_state_norm_sq": (C.c_int, [_vp, _P(_dbl)]),
    "rq_qaoa_batch_create": (C.c_int, [_u32, _P(_u32), _P(_u32), _P(_u32), _u32, _i32, _P(_vp)]),
    "rq_qaoa_batch_run": (C.c_int, [_vp, _u32, _P(_dbl), _P(_dbl), _P(_dbl), _u32, _u64, _P(_u64), _P(_u32)]),
    "rq_qaoa_batch_state": (C.c_int, [_vp, _u64, _P(_dbl)]),
    "rq_qaoa_batch_optimize": (C.c_int, [_vp, _u32, _dbl, _P(_dbl), _P(_dbl), _P(_dbl), _dbl, C.c_int32, _P(_dbl),
                                         _P(_u32)]),
    "rq_qaoa_batch_gradient": (C.c_int, [_vp, _P(_dbl), _P(_dbl), _P(_dbl), _P(_dbl)]),
    "rq_qaoa_batch_optimize_precond": (C.c_int, [_vp, _u32, _P(_dbl), _dbl, _P(_dbl), _P(_dbl), _P(_dbl), _dbl,
                                                 _P(_dbl), _P(_u32)]),
    "rq_qaoa_batch_set_convergence": (C.c_int, [_vp, _dbl]),
    "rq_qaoa_batch_last_ms": (C.c_int, [_vp, _P(C.c_float)]),
    "rq_qaoa_batch_last_profile": (C.c_int, [_vp, _P(_dbl)]),
    "rq_qaoa_batch_set_graphs": (C.c_int, [_vp, _i32]),
    "rq_qaoa_batch_last_graph": (C.c_int, [_vp, _P(_i32), _P(_u64)]),
    "rq_vqe_batch_set_graphs": (C.c_int, [_vp, _i32]),
    "rq_vqe_batch_last_graph": (C.c_int, [_vp, _P(_i32), _P(_u64)]),
    "rq_qaoa_batch_set_state_budget": (C.c_int, [_vp, _u64]),
    "rq_qaoa_batch_destroy": (C.c_int, [_vp]),
    "rq_vqe_batch_create": (C.c_int, [_u32, _u32, _P(_dbl), _P(RqPauliOp), _P(_u32), _u32, _i32, _P(_vp)]),
    "rq_vqe_batch_run": (C.c_int, [_vp, _u32, _P(_dbl), _i32, _P(_dbl), _P(_dbl)]),
    "rq_vqe_batch_last_ms": (C.c_int, [_vp, _P(C.c_float)]),
    "rq_vqe_batch_last_profile": (C.c_int, [_vp, _P(_dbl)]),
    "rq_vqe_batch_destroy": (C.c_int, [_vp]),
    "rq_gemm_bf16": (C.c_int, [_P(C.c_uint16), _P(C.c_uint16), _i32, _i32, _i32, _P(C.c_float)]),
    "rq_mlp_create": (C.c_int, [_i32, _i32, _i32, _i32, _u64, _P(_vp)]),
    "rq_mlp_destroy": (C.c_int, [_vp]),
    "rq_mlp_num_params": (C.c_int, [_vp, _P(C.c_int64)]),
    "rq_mlp_get_params": (C.c_int, [_vp, _P(C.c_float)]),
    "rq_mlp_set_params": (C.c_int, [_vp, _P(C.c_float)]),
    "rq_mlp_forward": (C.c_int, [_vp, _P(C.c_float), _i32, _P(C.c_float)]),
    "rq_mlp_gradients": (C.c_int, [_vp, _P(C.c_float), _P(C.c_float), _i32, _P(C.c_float), _P(C.c_float)]),
    "rq_mlp_train": (C.c_int, [_vp, _P(C.c_float), _P(C.c_float), _i32, _i32, _i32, C.c_float, _P(C.c_float)]),
    "rq_expectation_batch_noalloc": (C.c_int, [_vp, _u32, _i32, _P(RqPauliOp), _P(_u32), _u32, _P(_dbl), _vp]),
    "rq_state_normalize": (C.c_int, [_vp]),
    "rq_state_fidelity": (C.c_int, [_vp, _vp, _P(_dbl)]),
    "rq_state_download": (C.c_int, [_vp, _P(_dbl)]),
    "rq_state_upload": (C.c_int, [_vp, _P(_dbl)]),
}


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: the CUDA library is the only compute path of ruqu_b200. "
            "Build it with `python ruqu_b200/build.py`.")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    return lib.rq_last_error_message().decode(errors="replace")
