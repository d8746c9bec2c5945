"""Bounded device waits that run out (needs a GPU).

Every tensor-core kernel polls its mbarriers a bounded number of times.  Here
the limit is set to zero polls (rq_debug_set_wait_limit), so the first wait of
every CTA expires at once: the kernel must record the expiry, wait (with the
default limit) for the copies and MMAs it already started, free its tensor
memory and return -- no fault, no hang.  The host then sees RQ_ERR_TIMEOUT at
the next read-back, the flag is cleared, and with the default limit restored
the same handle and plan compute the right amplitudes again (1e-5 against the
oracle).  Nothing here faults or stalls the GPU: the waits end by their limit.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import ruqu_b200 as rq
from ruqu_b200 import _capi, workloads

pytestmark = pytest.mark.gpu

DEFAULT = 0xFFFFFFFF


@pytest.mark.parametrize("mode,lq", [(rq.RQ_EXEC_SWEEP_TC, 0), (rq.RQ_EXEC_SWEEP_TC16, 0),
                                     (rq.RQ_EXEC_SWEEP_TC16, 12)])
def test_sweep_wait_expiry_reports_timeout_and_state_recovers(mode, lq):
    """lq 0 = the default tile (13 local qubits here); 12 = the FP16 kernel's one-buffer,
    four-CTAs-per-SM instantiation, whose next image copy is issued after the MMAs."""
    n = 15
    gates = workloads.random_layer_circuit(n, 4, 7)
    st = rq.QuantumState(n, 0, "f32")
    plan = rq.Plan(st, gates, mode, local_qubits=lq) if lq else rq.Plan(st, gates, mode)
    assert plan.stats()["dense_ops"] > 0
    if lq:
        assert plan.stats()["local_qubits"] == lq
    st.synchronize()
    assert _capi.lib.rq_debug_set_wait_limit(0) == 0
    try:
        assert _capi.lib.rq_plan_execute(st.handle, plan._h) == _capi.RQ_OK
        rc = _capi.lib.rq_state_synchronize(st.handle)
    finally:
        assert _capi.lib.rq_debug_set_wait_limit(DEFAULT) == 0
    assert rc == _capi.RQ_ERR_TIMEOUT, (rc, _capi.last_error())
    assert "expired" in _capi.last_error()
    # the flag was cleared by the read-back that reported it; the handle works again
    assert _capi.lib.rq_state_synchronize(st.handle) == _capi.RQ_OK
    st.reset()
    plan.execute(st)
    ref = oracle.OracleState(n, oracle.RQ_F64, 0)
    ref.apply(gates)
    assert float(np.max(np.abs(st.state_vector() - ref.amplitudes()))) < 1e-5


def test_gemm_wait_expiry_reports_timeout_and_recovers():
    M, N, K = 128, 64, 128
    r = np.random.default_rng(1)
    a = r.integers(0, 1 << 16, size=(M, K), dtype=np.uint16) & 0x3FFF   # finite bf16 values
    b = r.integers(0, 1 << 16, size=(N, K), dtype=np.uint16) & 0x3FFF
    out = np.zeros((M, N), dtype=np.float32)

    def call():
        return _capi.lib.rq_gemm_bf16(a.ctypes.data_as(C.POINTER(C.c_uint16)),
                                      b.ctypes.data_as(C.POINTER(C.c_uint16)), M, N, K,
                                      out.ctypes.data_as(C.POINTER(C.c_float)))
    assert _capi.lib.rq_debug_set_wait_limit(0) == 0
    try:
        rc = call()
    finally:
        assert _capi.lib.rq_debug_set_wait_limit(DEFAULT) == 0
    assert rc == _capi.RQ_ERR_TIMEOUT, (rc, _capi.last_error())
    assert call() == _capi.RQ_OK, _capi.last_error()
    fa = (a.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    fb = (b.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    ref = fa @ fb.T
    assert float(np.max(np.abs(out - ref))) <= 2e-3 * float(np.max(np.abs(ref))) + 1e-30
