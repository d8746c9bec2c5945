"""The allocation-free expectation entry point (rq_expectation_batch_noalloc).

Callers whose device memory is fixed in advance, or owned by another
framework's allocator, cannot let the library call cudaMalloc.  This entry
point reads a caller-owned amplitude buffer and keeps its partial sums in one
static device array, so it allocates nothing.  These tests call it through the
C ABI, twice in a row with different Pauli strings, and compare each result with
the allocating entry point (rq_state_expectation_batch) on the same state.
The file sorts last so a failure here never hides the other GPU tests.
"""
import ctypes as C

import numpy as np
import pytest

from ruqu_b200 import QuantumState, _capi, workloads
from ruqu_b200.state import pauli_array

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-10, "f32": 1e-5}


def _strings(n, count, seed):
    r = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        k = int(r.integers(0, 6))
        out.append([(int(r.integers(0, n)), int(r.integers(0, 4))) for _ in range(k)])
    return out


def _noalloc(ptr, n, prec, strings, stream):
    arr, off = pauli_array(strings)
    out = np.full(len(strings), np.nan)
    rc = _capi.lib.rq_expectation_batch_noalloc(
        C.c_void_p(ptr), n, _capi.RQ_F32 if prec == "f32" else _capi.RQ_F64, arr,
        off.ctypes.data_as(C.POINTER(C.c_uint32)), len(strings),
        out.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(stream))
    return rc, out


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_noalloc_matches_allocating_entry_point(prec):
    n = 16
    st = QuantumState(n, 0, prec)
    st.apply_gates(workloads.random_layer_circuit(n, 4, 3))
    ptr, stream = st.device_pointer()
    st.synchronize()
    first = _strings(n, 100, 1) + [[], [(0, 2), (0, 2)]]
    second = _strings(n, 128, 2)
    rc1, got1 = _noalloc(ptr, n, prec, first, stream)
    rc2, got2 = _noalloc(ptr, n, prec, second, stream)
    assert rc1 == 0 and rc2 == 0, _capi.last_error()
    want1 = st.expectation_values(first)
    want2 = st.expectation_values(second)
    assert np.max(np.abs(got1 - want1)) < TOL[prec]
    assert np.max(np.abs(got2 - want2)) < TOL[prec]
    # the shared scratch keeps the previous call's partials; a repeat must not see them
    rc3, got3 = _noalloc(ptr, n, prec, first[:7], stream)
    assert rc3 == 0 and np.max(np.abs(got3 - want1[:7])) < TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n", [1, 2])
def test_noalloc_small_states_where_most_blocks_get_no_work(prec, n):
    """With 2 or 4 amplitudes nearly every reduction block has no element: each still
    writes a zero partial, so the sums never pick up what an earlier call left in the
    shared scratch (a 16-qubit call first fills it with non-zero partials)."""
    big = QuantumState(16, 0, prec)
    big.apply_gates(workloads.random_layer_circuit(16, 2, 4))
    bptr, bstream = big.device_pointer()
    big.synchronize()
    fill = _strings(16, 64, 5)
    rc0, _ = _noalloc(bptr, 16, prec, fill, bstream)
    assert rc0 == 0, _capi.last_error()
    st = QuantumState(n, 0, prec)
    st.apply_gates([(9, 0, 0, 0.7), (10, n - 1, 0, 1.3)])   # Ry(0.7) q0, Rz(1.3) q(n-1)
    ptr, stream = st.device_pointer()
    st.synchronize()
    strings = [[], [(0, 3)], [(0, 1)], [(0, 2)], [(n - 1, 3)], [(0, 1), (n - 1, 3)]]
    for _ in range(2):
        rc, got = _noalloc(ptr, n, prec, strings, stream)
        assert rc == 0, _capi.last_error()
        want = st.expectation_values(strings)
        assert np.max(np.abs(got - want)) < TOL[prec]


def test_noalloc_rejects_null_ops_for_non_empty_strings():
    n = 4
    st = QuantumState(n, 0, "f64")
    ptr, stream = st.device_pointer()
    st.synchronize()
    off = np.array([0, 1], dtype=np.uint32)
    out = np.full(1, np.nan)
    rc = _capi.lib.rq_expectation_batch_noalloc(
        C.c_void_p(ptr), n, _capi.RQ_F64, None, off.ctypes.data_as(C.POINTER(C.c_uint32)), 1,
        out.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(stream))
    assert rc == _capi.RQ_ERR_INVALID_ARGUMENT
    assert np.isnan(out).all()


def test_noalloc_rejects_more_strings_than_its_scratch_holds():
    n = 10
    st = QuantumState(n, 0, "f64")
    ptr, stream = st.device_pointer()
    st.synchronize()
    limit = 128
    rc, out = _noalloc(ptr, n, "f64", _strings(n, limit + 1, 3), stream)
    assert rc == _capi.RQ_ERR_INVALID_ARGUMENT
    assert str(limit) in _capi.last_error()
    assert np.isnan(out).all()
