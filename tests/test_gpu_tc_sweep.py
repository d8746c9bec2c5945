"""Tensor-core sweeps (RQ_EXEC_SWEEP_TC / _FAST / _TC16) vs the oracle (needs a GPU).

Each phase's slot-local gate run is one dense 32x32 complex unitary applied on
the tensor cores: as 3xTF32 MMAs (RQ_EXEC_SWEEP_TC), one TF32 pass (_FAST), or
three FP16 passes of per-tile-scaled high/low splits (_TC16).  3xTF32 and the
FP16 split keep FP32-level accuracy: amplitudes max-abs 1e-5 against the
oracle's f64 state (the f32 bar), as the CUDA-core sweep.  One TF32 pass
carries 10-bit operand mantissas: its bar is 1e-4 max-abs at up to 20 qubits,
and the norm stays within 1e-3.
"""
import math

import numpy as np
import pytest

import oracle
import ruqu_b200 as rq
from ruqu_b200 import QuantumState, workloads

pytestmark = pytest.mark.gpu

ONE_Q = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11]
TWO_Q = [12, 13, 14, 15]


def _mixed_circuit(n, ngates, seed):
    r = np.random.default_rng(seed)
    out = []
    for _ in range(ngates):
        k = int(r.choice(ONE_Q + TWO_Q))
        a = int(r.integers(0, n))
        b = int((a + 1 + r.integers(0, n - 1)) % n)
        out.append((k, a, b if k in TWO_Q else 0, float(r.uniform(0, 2 * math.pi))))
    return out


def _oracle_f64(n, gates):
    o = oracle.OracleState(n, oracle.RQ_F64, 0)
    o.apply(gates)
    return o.amplitudes()


MODES = [rq.RQ_EXEC_SWEEP_TC, rq.RQ_EXEC_SWEEP_TC16]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("n", [12, 13, 14, 17])
def test_tc_random_layers_match_oracle(n, mode):
    gates = workloads.random_layer_circuit(n, 8, n)
    ref = _oracle_f64(n, gates)
    g = QuantumState(n, 0, "f32")
    plan = rq.Plan(g, gates, mode)
    st = plan.stats()
    assert st["dense_ops"] > 0
    plan.execute(g)
    err = float(np.max(np.abs(g.state_vector() - ref)))
    assert err < 1e-5, err


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("n", [12, 15, 18])
def test_tc_mixed_gates_match_oracle(n, mode):
    """Every gate kind, controls and diagonals on thread bits (deferred past the dense op)."""
    gates = _mixed_circuit(n, 400, 100 + n)
    ref = _oracle_f64(n, gates)
    g = QuantumState(n, 0, "f32")
    g.apply_gates(gates, mode)
    assert float(np.max(np.abs(g.state_vector() - ref))) < 1e-5


def test_tc_fast_20q_random_layers():
    n = 20
    gates = workloads.random_layer_circuit(n, 40, 0)
    ref = _oracle_f64(n, gates)
    g = QuantumState(n, 0, "f32")
    g.apply_gates(gates, rq.RQ_EXEC_SWEEP_TC_FAST)
    v = g.state_vector()
    assert float(np.max(np.abs(v - ref))) < 1e-4
    assert abs(float(np.vdot(v, v).real) - 1.0) < 1e-3
    h = QuantumState(n, 0, "f32")
    h.apply_gates(gates, rq.RQ_EXEC_SWEEP_TC)
    assert float(np.max(np.abs(h.state_vector() - ref))) < 1e-5


def test_tc16_20q_random_layers_config1_circuit():
    """The 20-qubit, 40-layer, seed-0 random-layer circuit on complex f32 with the FP16-split
    dense ops: max-abs 1e-5 against the oracle's f64 amplitudes, norm within 1e-5."""
    n = 20
    gates = workloads.random_layer_circuit(n, 40, 0)
    ref = _oracle_f64(n, gates)
    g = QuantumState(n, 0, "f32")
    plan = rq.Plan(g, gates, rq.RQ_EXEC_SWEEP_TC16)
    assert plan.stats()["dense_ops"] > 0
    plan.execute(g)
    v = g.state_vector()
    assert float(np.max(np.abs(v - ref))) < 1e-5
    assert abs(float(np.vdot(v, v).real) - 1.0) < 1e-5


def test_tc16_scales_each_tile_unnormalised_and_tiny_tiles():
    """The FP16 split scales every tile by a power of two from its norm: a state of norm 40
    (amplitudes far outside the FP16 range once scaled for a unit state) and a state whose
    upper half is 1e-30 of its lower half both keep FP32-level relative accuracy."""
    n = 16
    gates = workloads.random_layer_circuit(n, 6, 9)
    r = np.random.default_rng(3)
    for kind in ("large", "tiny"):
        a = r.normal(size=1 << n) + 1j * r.normal(size=1 << n)
        a /= np.linalg.norm(a)
        if kind == "large":
            a *= 40.0
        else:
            a[1 << (n - 1):] *= 1e-30
        o = oracle.OracleState.from_amplitudes(a, n, oracle.RQ_F64)
        o.apply(gates)
        ref = o.amplitudes()
        g = QuantumState.from_amplitudes(a, n, "f32")
        g.apply_gates(gates, rq.RQ_EXEC_SWEEP_TC16)
        v = g.state_vector()
        scale = float(np.max(np.abs(ref)))
        assert float(np.max(np.abs(v - ref))) < 1e-5 * scale, kind
        if kind == "tiny":   # the tiles of the small half, relative to their own size
            lo = slice(1 << (n - 1), None)
            assert float(np.max(np.abs(v[lo] - ref[lo]))) < 1e-5 * float(np.max(np.abs(ref[lo])))


@pytest.mark.parametrize("mode", MODES)
def test_tc_plan_replays_and_equals_cuda_sweep_24q(mode):
    n = 24
    gates = workloads.random_layer_circuit(n, 6, 5)
    a = QuantumState(n, 0, "f32")
    b = QuantumState(n, 0, "f32")
    pa = rq.Plan(a, gates, rq.RQ_EXEC_SWEEP)
    pb = rq.Plan(b, gates, mode)
    for _ in range(2):
        a.reset()
        b.reset()
        pa.execute(a)
        pb.execute(b)
    assert np.max(np.abs(a.state_vector() - b.state_vector())) < 1e-5


def test_repeated_gate_lists_reuse_their_program_and_changes_are_seen():
    """apply_gates keeps the prepared programs of recent gate lists: the same list again gives
    the same amplitudes, and a list that differs in one angle is planned afresh."""
    n = 14
    gates = workloads.random_layer_circuit(n, 4, 2)
    g = QuantumState(n, 0, "f32")
    g.apply_gates(gates, rq.RQ_EXEC_SWEEP_TC)
    first = g.state_vector()
    g.reset()
    g.apply_gates(gates, rq.RQ_EXEC_SWEEP_TC)
    assert np.array_equal(first, g.state_vector())
    changed = list(gates)
    k = next(i for i, x in enumerate(changed) if x[0] in (9, 10))   # an Rx / Ry / Rz angle
    kind, a, b, ang = changed[k]
    changed[k] = (kind, a, b, ang + 0.3)
    g.reset()
    g.apply_gates(changed, rq.RQ_EXEC_SWEEP_TC)
    ref = _oracle_f64(n, changed)
    assert float(np.max(np.abs(g.state_vector() - ref))) < 1e-5


@pytest.mark.parametrize("prec,mode", [("f64", rq.RQ_EXEC_SWEEP), ("f32", rq.RQ_EXEC_SWEEP), ("f32", rq.RQ_EXEC_SWEEP_TC),
                                       ("f32", rq.RQ_EXEC_SWEEP_TC16), ("f64", rq.RQ_EXEC_PER_GATE)])
def test_plan_update_equals_a_fresh_plan(prec, mode):
    """rq_plan_update: a plan built for one angle set and given another (same kinds and qubits)
    computes exactly what a plan built for the new angles computes (bit for bit: the fused
    matrices are re-derived the same way and the operand images are built by the same GPU
    kernel), and matches the oracle (1e-12 f64, 1e-5 f32)."""
    n = 16
    a = workloads.random_layer_circuit(n, 6, 21)
    b = workloads.random_layer_circuit(n, 6, 22)   # same structure, new angles
    sa = QuantumState(n, 0, prec)
    plan = rq.Plan(sa, a, mode)
    plan.execute(sa)
    plan.update(sa, b)
    sa.reset()
    plan.execute(sa)
    got = sa.state_vector()
    sb = QuantumState(n, 0, prec)
    fresh = rq.Plan(sb, b, mode)
    fresh.execute(sb)
    assert np.array_equal(got, sb.state_vector())
    tol = 1e-12 if prec == "f64" else 1e-5
    assert float(np.max(np.abs(got - _oracle_f64(n, b)))) < tol


def test_plan_update_rejects_another_structure_and_keeps_the_plan():
    n = 14
    a = workloads.random_layer_circuit(n, 4, 5)
    other = list(a)
    k = next(i for i, g in enumerate(other) if g[0] == 12)   # move one CNOT
    other[k] = (12, other[k][1], (other[k][2] + 1) % n if (other[k][2] + 1) % n != other[k][1] else (other[k][2] + 2) % n, 0.0)
    s = QuantumState(n, 0, "f32")
    plan = rq.Plan(s, a, rq.RQ_EXEC_SWEEP_TC16)
    with pytest.raises(rq.CircuitError):
        plan.update(s, other)
    with pytest.raises(rq.CircuitError):
        plan.update(s, a[:-1])
    plan.execute(s)
    assert float(np.max(np.abs(s.state_vector() - _oracle_f64(n, a)))) < 1e-5


def test_apply_with_new_angles_reuses_the_structure_across_states_and_streams():
    """apply_gates keeps recent plans by structure: new angles rebuild only the tables, in
    stream order; two states (two streams) alternating between angle sets both stay exact."""
    n = 15
    sets = [workloads.random_layer_circuit(n, 5, 40 + k) for k in range(4)]
    refs = [_oracle_f64(n, g) for g in sets]
    s1, s2 = QuantumState(n, 0, "f32"), QuantumState(n, 0, "f32")
    for rounds in range(2):
        for k, g in enumerate(sets):
            st = s1 if k % 2 == 0 else s2
            st.reset()
            st.apply_gates(g, rq.RQ_EXEC_SWEEP_TC16)
            assert float(np.max(np.abs(st.state_vector() - refs[k]))) < 1e-5, (rounds, k)


def test_tc16_non_unitary_matrices_run_on_the_tf32_split():
    """A Unitary1Q matrix that is not unitary (a scaled projector, a general 2x2) breaks the
    FP16-split sweep's tile bound and norm restoration, so such lists plan as 3xTF32 sweeps
    (also under RQ_EXEC_SWEEP_TC16), a TC16 plan refuses such values in rq_plan_update, and
    apply_gates re-plans them; every result matches the oracle (1e-5 of the largest
    amplitude)."""
    n = 14
    base = workloads.random_layer_circuit(n, 4, 7)
    had = [2 ** -0.5, 0.0, 2 ** -0.5, 0.0, 2 ** -0.5, 0.0, -(2 ** -0.5), 0.0]
    proj = [3.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0]
    gen = [0.3, 0.1, 1.2, -0.4, 0.0, 0.7, 0.9, 0.2]
    unit = base[:40] + [(19, 3, 0, 0.0, had), (19, 9, 0, 0.0, had)] + base[40:]
    nonu = base[:40] + [(19, 3, 0, 0.0, proj), (19, 9, 0, 0.0, gen)] + base[40:]

    def err(g, gates):
        ref = _oracle_f64(n, gates)
        return float(np.max(np.abs(g.state_vector() - ref))) / max(1.0, float(np.max(np.abs(ref))))

    g = QuantumState(n, 0, "f32")
    plan = rq.Plan(g, nonu, rq.RQ_EXEC_SWEEP_TC16)
    assert plan.stats()["exec_mode"] == rq.RQ_EXEC_SWEEP_TC
    plan.execute(g)
    assert err(g, nonu) < 1e-5
    g.reset()
    p16 = rq.Plan(g, unit, rq.RQ_EXEC_SWEEP_TC16)
    assert p16.stats()["exec_mode"] == rq.RQ_EXEC_SWEEP_TC16
    with pytest.raises(rq.CircuitError):
        p16.update(g, nonu)
    p16.execute(g)
    assert err(g, unit) < 1e-5
    for gates in (unit, nonu, unit):   # the apply path: structure match, then a fresh plan
        g.reset()
        g.apply_gates(gates, rq.RQ_EXEC_SWEEP_TC16)
        assert err(g, gates) < 1e-5


@pytest.mark.parametrize("n,layers,lq", [(14, 6, 14), (17, 8, 14), (20, 10, 14), (22, 8, 12)])
def test_tc16_12_and_14_qubit_tiles_match_oracle(n, layers, lq):
    """FP16-split sweeps on 14-qubit tiles (one 512-thread CTA per SM, four 128-row halves,
    a ninth thread bit in the shared-memory layout) and on 12-qubit tiles (four 128-thread
    CTAs per SM with one operand-image buffer; at 22 qubits 1024 tiles over at most 592 CTAs,
    so CTAs copy the next tile's first image after their last phase): amplitudes within 1e-5
    of the f64 oracle, fewer (14) or more (12) sweeps than 13-qubit tiles, and a rebind to new
    angles equals a fresh plan."""
    gates = workloads.random_layer_circuit(n, layers, 30 + n)
    g = QuantumState(n, 0, "f32")
    plan = rq.Plan(g, gates, rq.RQ_EXEC_SWEEP_TC16, local_qubits=lq)
    st = plan.stats()
    assert st["local_qubits"] == lq and st["exec_mode"] == rq.RQ_EXEC_SWEEP_TC16
    plan.execute(g)
    assert float(np.max(np.abs(g.state_vector() - _oracle_f64(n, gates)))) < 1e-5
    if n >= 17:
        p13 = rq.Plan(QuantumState(n, 0, "f32"), gates, rq.RQ_EXEC_SWEEP_TC16, local_qubits=13)
        if lq == 14:
            assert st["sweeps"] <= p13.stats()["sweeps"]
        else:
            assert st["sweeps"] >= p13.stats()["sweeps"]
    new = workloads.random_layer_circuit(n, layers, 31 + n)
    plan.update(g, new)
    g.reset()
    plan.execute(g)
    f = QuantumState(n, 0, "f32")
    rq.Plan(f, new, rq.RQ_EXEC_SWEEP_TC16, local_qubits=lq).execute(f)
    assert np.array_equal(g.state_vector(), f.state_vector())


def test_tiled_plan_rejects_bad_tile_sizes():
    g = QuantumState(16, 0, "f32")
    gates = workloads.random_layer_circuit(16, 2, 1)
    for mode, lq in ((rq.RQ_EXEC_SWEEP_TC, 14), (rq.RQ_EXEC_SWEEP_TC16, 15), (rq.RQ_EXEC_SWEEP_TC16, 11),
                     (rq.RQ_EXEC_SWEEP, 13)):
        with pytest.raises(rq.InvalidArgument):
            rq.Plan(g, gates, mode, local_qubits=lq)
    with pytest.raises(rq.InvalidArgument):
        rq.Plan(QuantumState(16, 0, "f64"), gates, rq.RQ_EXEC_SWEEP_TC16, local_qubits=13)
