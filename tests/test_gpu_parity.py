"""CUDA path vs the oracle, through the C ABI (needs a GPU).

Tolerances: amplitudes max-abs 1e-12 for complex f64 states and 1e-5 for
complex f32 states (at up to 20 qubits); expectation values and energies
1e-10 absolute for f64 and 1e-5 for f32 (FP64 accumulation on the device);
shot bitstrings, cut values and histograms bit-exact.
"""
import math
import os

import numpy as np
import pytest

import oracle
import ruqu_b200 as rq
from golden.reference_kats import CASES, EPS, FIDELITY
from kat_runner import GpuBackend, run_case
from ruqu_b200 import QuantumState, workloads
from ruqu_b200.qaoa import Graph, QaoaConfig, run_qaoa
from ruqu_b200.vqe import VqeConfig, h2_hamiltonian, run_vqe

pytestmark = pytest.mark.gpu

H, X, Y, Z, S, SDG, T, TDG, RX, RY, RZ, PHASE, CNOT, CZ, SWAP, RZZ, MEAS, RESET, BARRIER, U1 = range(20)
PREC = {"f64": oracle.RQ_F64, "f32": oracle.RQ_F32}
TOL = {"f64": 1e-12, "f32": 1e-5}
MODES = [rq.RQ_EXEC_PER_GATE, rq.RQ_EXEC_SWEEP]


def _random_state(n, seed):
    r = np.random.default_rng(seed)
    a = r.normal(size=1 << n) + 1j * r.normal(size=1 << n)
    return a / np.linalg.norm(a)


def _pair(n, prec, seed=0, amps=None):
    """(GPU state, oracle state) holding the same amplitudes."""
    if amps is None:
        return QuantumState(n, seed, prec), oracle.OracleState(n, PREC[prec], seed)
    g = QuantumState.from_amplitudes(amps, n, prec, seed)
    o = oracle.OracleState.from_amplitudes(amps, n, PREC[prec], seed)
    return g, o


def _maxdiff(g, o):
    return float(np.max(np.abs(g.state_vector() - o.amplitudes())))


# ---------------------------------------------------------------- reference KATs
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_reference_kats_on_gpu(case, prec):
    run_case(GpuBackend(case["n"], PREC[prec]), case, EPS if prec == "f64" else 1e-5)


@pytest.mark.parametrize("fk", FIDELITY, ids=[f["ref"] for f in FIDELITY])
def test_fidelity_kats_on_gpu(fk):
    a = QuantumState(fk["n"])
    b = QuantumState(fk["n"])
    if fk["a"]:
        a.apply_gates([s[1:] for s in fk["a"]])
    if fk["b"]:
        b.apply_gates([s[1:] for s in fk["b"]])
    assert abs(a.fidelity(b) - fk["value"]) < EPS


# ---------------------------------------------------------------- every gate x every qubit
ONE_Q = [H, X, Y, Z, S, SDG, T, TDG, RX, RY, RZ, PHASE]
TWO_Q = [CNOT, CZ, SWAP, RZZ]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("mode", MODES)
def test_every_gate_every_qubit(prec, mode):
    n = 8
    amps = _random_state(n, 1)
    for kind in ONE_Q:
        for q in range(n):
            g, o = _pair(n, prec, amps=amps)
            gate = [(kind, q, 0, 0.7 + 0.1 * q)]
            g.apply_gates(gate, mode)
            o.apply(gate)
            assert _maxdiff(g, o) < TOL[prec], (kind, q)
    for kind in TWO_Q:
        for a in range(n):
            for b in range(n):
                if a == b:
                    continue
                g, o = _pair(n, prec, amps=amps)
                gate = [(kind, a, b, 1.1 + 0.05 * a - 0.03 * b)]
                g.apply_gates(gate, mode)
                o.apply(gate)
                assert _maxdiff(g, o) < TOL[prec], (kind, a, b)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_unitary1q_and_matrix_entry_points(prec):
    n = 9
    amps = _random_state(n, 2)
    th, ph, la = 0.3, 1.2, -0.4
    u = np.array([[math.cos(th / 2), -np.exp(1j * la) * math.sin(th / 2)],
                  [np.exp(1j * ph) * math.sin(th / 2), np.exp(1j * (ph + la)) * math.cos(th / 2)]])
    m8 = [v for c in u.reshape(-1) for v in (c.real, c.imag)]
    for q in range(n):
        g, o = _pair(n, prec, amps=amps)
        g.apply_gates([(U1, q, 0, 0.0, m8)], rq.RQ_EXEC_SWEEP)
        o.apply([(U1, q, 0, 0.0, m8)])
        assert _maxdiff(g, o) < TOL[prec]
        g, o = _pair(n, prec, amps=amps)
        g.apply_single_qubit_gate(q, u)
        o.apply_1q_matrix(q, m8)
        assert _maxdiff(g, o) < TOL[prec]
    r = np.random.default_rng(3)
    m4 = np.linalg.qr(r.normal(size=(4, 4)) + 1j * r.normal(size=(4, 4)))[0]
    m32 = [v for c in m4.reshape(-1) for v in (c.real, c.imag)]
    for a, b in ((0, 1), (1, 0), (2, 7), (8, 3)):
        g, o = _pair(n, prec, amps=amps)
        g.apply_two_qubit_gate(a, b, m4)
        o.apply_2q_matrix(a, b, m32)
        assert _maxdiff(g, o) < TOL[prec]


# ---------------------------------------------------------------- random circuits
def _mixed_circuit(n, ngates, seed):
    r = np.random.default_rng(seed)
    out = []
    for _ in range(ngates):
        k = int(r.choice(ONE_Q + TWO_Q))
        a = int(r.integers(0, n))
        b = int((a + 1 + r.integers(0, n - 1)) % n)
        out.append((k, a, b if k in TWO_Q else 0, float(r.uniform(0, 2 * math.pi))))
    return out


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("n", [7, 12, 16])
def test_random_mixed_circuits(n, mode, prec):
    gates = _mixed_circuit(n, 300, n)
    g, o = _pair(n, prec)
    g.apply_gates(gates, mode)
    o.apply(gates)
    assert _maxdiff(g, o) < TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_config1_random_layers_20q(prec):
    """20 qubits, 40 random layers, seed 0: amplitudes, <Z_i>, 4096 shots."""
    n, layers = 20, 40
    gates = workloads.random_layer_circuit(n, layers, 0)
    o = oracle.OracleState(n, oracle.RQ_F64, 0)
    o.apply(gates)
    ref = o.amplitudes()
    for mode in MODES:
        g = QuantumState(n, 0, prec)
        g.apply_gates(gates, mode)
        got = g.state_vector()
        err = float(np.max(np.abs(got - ref)))
        assert err < TOL[prec], (mode, err)
        z = g.expectation_values([[(q, 3)] for q in range(n)])
        zo = np.array([o.expectation([(q, 3)]) for q in range(n)])
        assert np.max(np.abs(z - zo)) < (1e-10 if prec == "f64" else 1e-5)
    # shots: bit-exact against the oracle's sampler fed the device state's probabilities
    bits = g.sample(4096, 42)
    pg = np.abs(got.real) ** 2 + np.abs(got.imag) ** 2
    pg = got.real * got.real + got.imag * got.imag
    assert (bits == oracle.tree_sample(pg, n, list(range(n)), 42, 4096)).all()
    if prec == "f64":
        # and against the oracle's own f64 state
        assert (bits == oracle.tree_sample(o.probabilities(), n, list(range(n)), 42, 4096)).all()


# ---------------------------------------------------------------- reductions
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_expectation_batches(prec):
    n = 14
    amps = _random_state(n, 4)
    g, o = _pair(n, prec, amps=amps)
    r = np.random.default_rng(5)
    strings = []
    for _ in range(60):
        k = int(r.integers(0, 5))
        strings.append([(int(r.integers(0, n)), int(r.integers(0, 4))) for _ in range(k)])
    strings += [[(0, 2), (0, 2)], [(3, 1), (3, 1), (5, 3)], [(2, 2), (2, 1)]]   # repeated qubits
    got = g.expectation_values(strings)
    want = np.array([o.expectation(s) for s in strings])
    tol = 1e-10 if prec == "f64" else 1e-5
    assert np.max(np.abs(got - want)) < tol
    coeffs = r.normal(size=len(strings))
    hg = g.expectation_hamiltonian(rq.Hamiltonian([(c, rq.PauliString(s)) for c, s in zip(coeffs, strings)], n))
    assert abs(hg - o.expectation_hamiltonian(coeffs, strings)) < 10 * tol
    for q in range(n):
        assert abs(g.probability_of_qubit(q) - o.probability_of_qubit(q)) < tol
    assert abs(g.norm_sq() - 1.0) < tol
    assert np.max(np.abs(g.probabilities() - o.probabilities())) < tol


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_normalize_and_fidelity(prec):
    n = 12
    a = _random_state(n, 6) * 3.0
    g, o = _pair(n, prec, amps=a)
    g.normalize()
    o.normalize()
    assert _maxdiff(g, o) < TOL[prec]
    b = _random_state(n, 7)
    g2, o2 = _pair(n, prec, amps=b)
    assert abs(g.fidelity(g2) - o.fidelity(o2)) < (1e-12 if prec == "f64" else 1e-5)
    assert abs(g.fidelity(g2) - g2.fidelity(g)) < 1e-12
    g3 = QuantumState(n - 1)
    assert g.fidelity(g3) == 0.0


# ---------------------------------------------------------------- measurement
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_measure_reset_sequences_match_oracle(prec):
    n = 10
    for seed in range(6):
        g, o = _pair(n, prec, seed=seed)
        prog = _mixed_circuit(n, 40, 100 + seed)
        prog[10:10] = [(MEAS, 3, 0, 0.0)]
        prog[25:25] = [(RESET, 5, 0, 0.0), (MEAS, 0, 0, 0.0)]
        prog += [(MEAS, q, 0, 0.0) for q in range(n)]
        mg = g.apply_gates(prog)
        mo = o.apply(prog)
        assert [(m.qubit, m.result) for m in mg] == [(q, r) for q, r, _ in mo]
        for m, (_, _, p) in zip(mg, mo):
            assert abs(m.probability - p) < (1e-9 if prec == "f64" else 1e-5)
        assert _maxdiff(g, o) < (1e-9 if prec == "f64" else 1e-5)


def test_run_shots_matches_literal_reference():
    for circ, n in (([(H, 0), (MEAS, 0)], 1),
                    ([(H, 0), (CNOT, 0, 1), (MEAS, 0), (MEAS, 1)], 2),
                    (_mixed_circuit(5, 30, 9), 5),
                    (_mixed_circuit(4, 20, 10) + [(MEAS, 2), (MEAS, 0), (MEAS, 2)], 4),
                    ([(H, 0), (MEAS, 0), (H, 1), (CNOT, 1, 2), (MEAS, 2)], 3)):   # mid-circuit: per-shot path
        c = rq.QuantumCircuit(n)
        for t in circ:
            c.add_gate(rq.Gate(t[0], t[1], t[2] if len(t) > 2 else 0, t[3] if len(t) > 3 else 0.0))
        res = rq.Simulator.run_shots(c, 300, 42)
        lit = oracle.run_shots_literal(n, circ, 300, 42)
        want = {}
        for v in lit.tolist():
            key = tuple(bool((v >> q) & 1) for q in range(n))
            want[key] = want.get(key, 0) + 1
        assert res.counts == want


def test_sampling_measurement_orders_exact():
    n = 11
    amps = _random_state(n, 8)
    g, _ = _pair(n, "f64", amps=amps)
    p = g.probabilities()
    for order in (list(range(n)), [3, 1, 4], [10, 0, 5, 5, 2], list(reversed(range(n)))):
        got = g.sample(2000, 1234, order)
        want = oracle.tree_sample(p, n, order, 1234, 2000)
        assert (got == want).all()


# ---------------------------------------------------------------- errors
def test_errors_and_validation_before_launch():
    with pytest.raises(rq.QubitLimitExceeded):
        QuantumState(35)
    with pytest.raises(rq.QubitLimitExceeded):
        QuantumState(34, precision="f32")
    with pytest.raises(rq.CircuitError):
        QuantumState(0)
    s = QuantumState(3)
    s.apply_gates([(H, 0)])
    before = s.state_vector()
    with pytest.raises(rq.InvalidQubitIndex):
        s.apply_gates([(X, 1), (H, 5)])        # whole list validated first: X not applied
    assert np.array_equal(s.state_vector(), before)
    with pytest.raises(rq.CircuitError):
        s.apply_gates([(CNOT, 1, 1)])
    with pytest.raises(rq.InvalidQubitIndex):
        s.expectation_value([(7, 3)])
    with pytest.raises(rq.InvalidStateVector):
        QuantumState.from_amplitudes(np.ones(5), 3)


# ---------------------------------------------------------------- drivers
def test_run_qaoa_matches_reference_driver():
    g = Graph.unweighted(4, [(0, 1), (1, 2), (2, 3), (0, 3)])
    r = run_qaoa(QaoaConfig(g, 2, 12, 0.1, 42))
    ro = oracle.run_qaoa(4, g.edges, 2, 12, 0.1)
    assert len(r.energy_history) == len(ro["history"])
    assert np.max(np.abs(np.array(r.energy_history) - ro["history"])) < 1e-9
    assert np.max(np.abs(np.array(r.optimal_gammas) - ro["gammas"])) < 1e-9
    idx = sum(int(b) << q for q, b in enumerate(r.best_bitstring))
    assert idx == ro["best_bits"]


def test_run_vqe_matches_reference_driver():
    h = h2_hamiltonian()
    r = run_vqe(VqeConfig(h, 2, 2, 15, 0.001, 0.1, 42))
    c = [t[0] for t in h.terms]
    terms = [[(q, int(o)) for q, o in t[1].ops] for t in h.terms]
    ro = oracle.run_vqe(2, 2, c, terms, 15, 0.001, 0.1)
    assert np.max(np.abs(np.array(r.energy_history) - ro["history"])) < 1e-9
    assert r.optimal_energy < -0.8 or len(r.energy_history) < 50


# ---------------------------------------------------------------- large-state properties
def test_sweep_equals_per_gate_24q_f32():
    n = 24
    gates = workloads.random_layer_circuit(n, 6, 5)
    a = QuantumState(n, 0, "f32")
    b = QuantumState(n, 0, "f32")
    a.apply_gates(gates, rq.RQ_EXEC_PER_GATE)
    b.apply_gates(gates, rq.RQ_EXEC_SWEEP)
    va, vb = a.state_vector(), b.state_vector()
    assert np.max(np.abs(va - vb)) < 1e-5
    assert abs(b.norm_sq() - 1) < 1e-4


class _DeviceArray:
    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def _device_amplitudes(state, n, prec):
    """The state's amplitudes as a complex torch tensor on the device (no host copy)."""
    import torch
    ptr, _ = state.device_pointer()
    state.synchronize()
    t = torch.as_tensor(_DeviceArray(ptr, 2 << n, "<f4" if prec == "f32" else "<f8"), device="cuda")
    return torch.view_as_complex(t.view(-1, 2))


def _golden_26q():
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "random_layers_26q_seed1.npz")
    return np.load(path)


@pytest.mark.parametrize("prec,mode", [("f64", rq.RQ_EXEC_SWEEP), ("f64", rq.RQ_EXEC_PER_GATE),
                                       ("f32", rq.RQ_EXEC_SWEEP_TC), ("f32", rq.RQ_EXEC_SWEEP_TC16)])
def test_26q_20_layers_against_oracle_fixture(prec, mode):
    """The config's oracle check at 26 qubits: the 20-layer, seed-1 random-layer circuit
    (1,300 gates) against the oracle's f64 state (tests/golden/random_layers_26q_seed1.npz,
    made by make_random_layers_26q.py): 16,384 sampled amplitudes, <Z_q> of every qubit and
    the norms of 256 blocks of 2^18 amplitudes.  Tolerances: f64 (CUDA-core sweeps and the
    unfused per-gate kernels) 1e-12 on amplitudes and 1e-10 on the sums; f32 through the
    tensor-core sweeps (3xTF32 and the FP16 split) 1e-5 on amplitudes and on the sums."""
    import torch
    f = _golden_26q()
    n, layers, seed = (int(x) for x in f["meta"])
    gates = workloads.random_layer_circuit(n, layers, seed)
    g = QuantumState(n, 0, prec)
    g.apply_gates(gates, mode)
    a = _device_amplitudes(g, n, prec)
    idx = torch.as_tensor(f["indices"], device="cuda")
    got = a[idx].to(torch.complex128).cpu().numpy()
    amp_tol, sum_tol = (1e-12, 1e-10) if prec == "f64" else (1e-5, 1e-5)
    assert float(np.max(np.abs(got - f["amps"]))) < amp_tol
    p = a.real.double() ** 2 + a.imag.double() ** 2
    blocks = p.view(256, -1).sum(dim=1).cpu().numpy()
    assert float(np.max(np.abs(blocks - f["blocks"]))) < sum_tol
    z = []
    for q in range(n):
        v = p.view(-1, 2, 1 << q)
        z.append(float(v[:, 0, :].sum() - v[:, 1, :].sum()))
    assert float(np.max(np.abs(np.array(z) - f["z"]))) < sum_tol


@pytest.mark.parametrize("mode", [rq.RQ_EXEC_SWEEP_TC, rq.RQ_EXEC_SWEEP_TC16])
def test_30q_tensor_core_f32_against_f64_sweep(mode):
    """The benchmark circuit itself (30 qubits, 20 layers, seed 1): the f32 tensor-core
    sweeps against the complex f64 CUDA-core sweep of the same circuit (the oracle would
    take hours at 2^30 amplitudes; the f64 sweep is pinned to it at 26 qubits above), max-abs
    over all 2^30 amplitudes below 1e-6; the norm within 1e-5 for the FP16 split (which
    restores each tile's norm) and 1e-4 for 3xTF32 (whose accumulation drifts ~5e-5 low over
    the 48 phases)."""
    import torch
    n, layers = 30, 20
    gates = workloads.random_layer_circuit(n, layers, 1)
    ref = QuantumState(n, 0, "f64")
    ref.apply_gates(gates, rq.RQ_EXEC_SWEEP)
    g = QuantumState(n, 0, "f32")
    g.apply_gates(gates, mode)
    a = _device_amplitudes(g, n, "f32")
    b = _device_amplitudes(ref, n, "f64")
    worst, norm = 0.0, 0.0
    chunk = 1 << 26
    for k in range(0, 1 << n, chunk):
        x = a[k:k + chunk].to(torch.complex128)
        worst = max(worst, float((x - b[k:k + chunk]).abs().max()))
        norm += float((x.real ** 2 + x.imag ** 2).sum())
    assert worst < 1e-6, worst
    assert abs(norm - 1.0) < (1e-5 if mode == rq.RQ_EXEC_SWEEP_TC16 else 1e-4), norm
