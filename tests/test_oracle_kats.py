"""Pins the CPU oracle against the reference's own known answers (no GPU).

The reference (Rust) cannot be built here, so the oracle (oracle/ruqu_oracle.cpp)
is a restatement; these tests tie it to every known-answer test the reference
holds for the path: crates/ruqu-core/tests/test_state.rs, test_simulator.rs,
test_gates.rs, mixed_precision.rs' unit tests, and the QAOA/VQE tests of
crates/ruqu-algorithms/tests/test_algorithms.rs.  The Philox stream is pinned
against the Random123 known-answer vectors.
"""
import math

import numpy as np
import pytest

import oracle
from golden.reference_kats import CASES, EPS, FIDELITY
from kat_runner import OracleBackend, run_case

H, X, Y, Z, S, SDG, T, TDG, RX, RY, RZ, PHASE, CNOT, CZ, SWAP, RZZ, MEAS, RESET, BARRIER, U1 = range(20)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_reference_kat_f64(case):
    run_case(OracleBackend(case["n"], oracle.RQ_F64), case, EPS)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_reference_kat_f32(case):
    # mixed_precision.rs:672-733 checks the f32 engine at 1e-5
    run_case(OracleBackend(case["n"], oracle.RQ_F32), case, 1e-5)


@pytest.mark.parametrize("fk", FIDELITY, ids=[f["ref"] for f in FIDELITY])
def test_fidelity_kats(fk):
    a = oracle.OracleState(fk["n"])
    b = oracle.OracleState(fk["n"])
    a.apply([s[1:] for s in fk["a"]])
    b.apply([s[1:] for s in fk["b"]])
    assert abs(a.fidelity(b) - fk["value"]) < EPS
    assert abs(a.fidelity(b) - b.fidelity(a)) < EPS   # test_state.rs:821-830


def test_philox_random123_known_answers():
    # Random123 kat_vectors for philox4x32_10
    assert list(oracle.philox([0, 0, 0, 0], [0, 0])) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert list(oracle.philox([0xffffffff] * 4, [0xffffffff] * 2)) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert list(oracle.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0])) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def _basis_apply(n, gates, idx):
    amps = np.zeros(1 << n, dtype=np.complex128)
    amps[idx] = 1
    s = oracle.OracleState.from_amplitudes(amps, n)
    s.apply(gates)
    return s.amplitudes()


def test_gate_matrices_columns():
    """Column k of each gate matrix = gate applied to |k> (test_gates.rs:89-640)."""
    s2 = 1 / math.sqrt(2)
    want = {
        H: [[s2, s2], [s2, -s2]],
        X: [[0, 1], [1, 0]],
        Y: [[0, -1j], [1j, 0]],
        Z: [[1, 0], [0, -1]],
        S: [[1, 0], [0, 1j]],
        T: [[1, 0], [0, complex(s2, s2)]],
        SDG: [[1, 0], [0, -1j]],
        TDG: [[1, 0], [0, complex(s2, -s2)]],
    }
    for kind, m in want.items():
        m = np.array(m, dtype=np.complex128)
        for col in range(2):
            out = _basis_apply(1, [(kind, 0)], col)
            assert np.allclose(out, m[:, col], atol=1e-12), kind
    for theta in (0.0, 0.3, math.pi / 2, math.pi, 2.5):
        c, s = math.cos(theta / 2), math.sin(theta / 2)
        rx = np.array([[c, -1j * s], [-1j * s, c]])
        ry = np.array([[c, -s], [s, c]])
        rz = np.diag([np.exp(-1j * theta / 2), np.exp(1j * theta / 2)])
        ph = np.diag([1, np.exp(1j * theta)])
        for kind, m in ((RX, rx), (RY, ry), (RZ, rz), (PHASE, ph)):
            for col in range(2):
                out = _basis_apply(1, [(kind, 0, 0, theta)], col)
                assert np.allclose(out, m[:, col], atol=1e-12), (kind, theta)


def test_two_qubit_matrix_conventions():
    """Row/column index = q1_bit*2 + q2_bit; CNOT(control, target) (test_gates.rs:464-640)."""
    def idx(b1, b2, q1, q2):
        return (b1 << q1) | (b2 << q2)
    for (q1, q2) in ((0, 1), (1, 0), (0, 2), (2, 1)):
        for b1 in (0, 1):
            for b2 in (0, 1):
                out = _basis_apply(3, [(CNOT, q1, q2)], idx(b1, b2, q1, q2))
                assert abs(out[idx(b1, b2 ^ b1, q1, q2)] - 1) < 1e-15
                out = _basis_apply(3, [(CZ, q1, q2)], idx(b1, b2, q1, q2))
                assert abs(out[idx(b1, b2, q1, q2)] - (-1 if b1 and b2 else 1)) < 1e-15
                out = _basis_apply(3, [(SWAP, q1, q2)], idx(b1, b2, q1, q2))
                assert abs(out[idx(b2, b1, q1, q2)] - 1) < 1e-15
                th = 0.77
                out = _basis_apply(3, [(RZZ, q1, q2, th)], idx(b1, b2, q1, q2))
                ph = np.exp(-1j * th / 2) if b1 == b2 else np.exp(1j * th / 2)
                assert abs(out[idx(b1, b2, q1, q2)] - ph) < 1e-15


def test_errors_mirror_quantum_error():
    with pytest.raises(oracle.OracleError) as e:
        oracle.OracleState(35)
    assert e.value.code == 1                     # QubitLimitExceeded (test_state.rs:859-862)
    with pytest.raises(oracle.OracleError) as e:
        oracle.OracleState(0)
    assert e.value.code == 5                     # CircuitError (test_state.rs:865-868)
    s = oracle.OracleState(2)
    with pytest.raises(oracle.OracleError) as e:
        s.apply([(H, 5)])
    assert e.value.code == 2                     # InvalidQubitIndex (mixed_precision.rs:736-741)
    with pytest.raises(oracle.OracleError) as e:
        s.apply([(CNOT, 1, 1)])
    assert e.value.code == 5                     # distinct qubits (state.rs:179-184)


def test_measurement_semantics():
    # |0> always measures 0, |1> always 1 (test_state.rs:457-471)
    s = oracle.OracleState(1, seed=7)
    assert s.measure(0)[1] is False
    s = oracle.OracleState(1, seed=7)
    s.apply([(X, 0)])
    q, r, p = s.measure(0)
    assert r is True and abs(p - 1) < 1e-12
    # collapse (test_state.rs:443-454)
    s = oracle.OracleState(1, seed=42)
    s.apply([(H, 0)])
    r = s.measure(0)[1]
    assert abs(s.probabilities()[1 if r else 0] - 1) < EPS
    # Bell measure_all agree (test_state.rs:474-482)
    for seed in range(20):
        s = oracle.OracleState(2, seed=seed)
        s.apply([(H, 0), (CNOT, 0, 1)])
        assert s.measure(0)[1] == s.measure(1)[1]
    # 200 seeds land 30-70% (test_state.rs:485-506)
    zeros = 0
    for seed in range(200):
        s = oracle.OracleState(1, seed=seed)
        s.apply([(H, 0)])
        zeros += not s.measure(0)[1]
    assert 0.3 < zeros / 200 < 0.7
    # same seed -> same outcome (test_state.rs:509-520)
    outs = []
    for _ in range(2):
        s = oracle.OracleState(1, seed=12345)
        s.apply([(H, 0)])
        outs.append(s.measure(0)[1])
    assert outs[0] == outs[1]


def test_teleportation():
    """test_state.rs:929-969: qubit 2 ends in Ry(1.23)|0> for every seed."""
    target = math.sin(1.23 / 2) ** 2
    for seed in (99, 1, 2, 3, 4):
        s = oracle.OracleState(3, seed=seed)
        s.apply([(RY, 0, 0, 1.23), (H, 1), (CNOT, 1, 2), (CNOT, 0, 1), (H, 0)])
        m0 = s.measure(0)[1]
        m1 = s.measure(1)[1]
        if m1:
            s.apply([(X, 2)])
        if m0:
            s.apply([(Z, 2)])
        assert abs(s.probability_of_qubit(2) - target) < 0.01


def test_run_shots_invariants():
    # X then measure -> all ones (test_simulator.rs:275-287)
    bits = oracle.run_shots_literal(1, [(X, 0), (MEAS, 0)], 100, 42)
    assert (bits == 1).all()
    # H measure ~50% (test_simulator.rs:289-309)
    bits = oracle.run_shots_literal(1, [(H, 0), (MEAS, 0)], 1000, 42)
    assert 0.4 < float((bits == 0).mean()) < 0.6
    # Bell never 01/10 (test_simulator.rs:311-332)
    bits = oracle.run_shots_literal(2, [(H, 0), (CNOT, 0, 1), (MEAS, 0), (MEAS, 1)], 500, 42)
    assert set(bits.tolist()) <= {0, 3}
    # seeded reproducibility (test_simulator.rs:334-343)
    a = oracle.run_shots_literal(1, [(H, 0), (MEAS, 0)], 100, 42)
    b = oracle.run_shots_literal(1, [(H, 0), (MEAS, 0)], 100, 42)
    assert (a == b).all()


def _random_circuit(n, ngates, rng):
    gates = []
    for _ in range(ngates):
        k = rng.integers(0, 16)
        q0 = int(rng.integers(0, n))
        q1 = int((q0 + 1 + rng.integers(0, n - 1)) % n) if n > 1 else 0
        if k in (CNOT, CZ, SWAP, RZZ) and n < 2:
            k = H
        gates.append((int(k), q0, q1 if k in (CNOT, CZ, SWAP, RZZ) else 0, float(rng.uniform(0, 2 * math.pi))))
    return gates


@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_tree_sampler_equals_literal_shots(n):
    """The prefix-tree sampler reproduces run_shots' per-shot collapse loop (simulator.rs:107-147) draw for draw."""
    rng = np.random.default_rng(n)
    for trial in range(3):
        gates = _random_circuit(n, 12, rng)
        lit = oracle.run_shots_literal(n, gates, 300, 1000 + trial)
        s = oracle.OracleState(n)
        s.apply(gates)
        tree = oracle.tree_sample(s.probabilities(), n, list(range(n)), 1000 + trial, 300)
        assert (lit == tree).all()
        # explicit measurement order (a permutation, with a repeat)
        order = list(rng.permutation(n)) + [int(rng.integers(0, n))]
        lit = oracle.run_shots_literal(n, gates + [(MEAS, int(q)) for q in order], 300, 77)
        tree = oracle.tree_sample(s.probabilities(), n, order, 77, 300)
        assert (lit == tree).all()


def test_parallel_kernels_match_scalar():
    rng = np.random.default_rng(5)
    gates = _random_circuit(12, 60, rng)
    a = oracle.OracleState(12)
    b = oracle.OracleState(12)
    a.apply(gates)
    b.apply(gates, parallel=True)
    assert np.max(np.abs(a.amplitudes() - b.amplitudes())) < 1e-12


def test_duplicate_pauli_qubits_quirk():
    """expectation_value reads each factor's bit from the original index (state.rs:366-395):
    a repeated Y on one qubit yields -<psi|psi>, repeated X or Z yield +1."""
    s = oracle.OracleState(2)
    s.apply([(H, 0), (RX, 1, 0, 0.4)])
    assert abs(s.expectation([(0, 2), (0, 2)]) + 1) < 1e-12
    assert abs(s.expectation([(0, 1), (0, 1)]) - 1) < 1e-12
    assert abs(s.expectation([(1, 3), (1, 3)]) - 1) < 1e-12


# ---- ruqu-algorithms behaviour (crates/ruqu-algorithms/tests/test_algorithms.rs) ----

def test_cut_values_exact():
    # test_algorithms.rs:616-671 and qaoa.rs:355-386
    tri = [(0, 1, 1.0), (1, 2, 1.0), (0, 2, 1.0)]
    probs = np.zeros(8)
    for bits, want in (((1, 0, 0), 2.0), ((0, 0, 0), 0.0), ((1, 1, 0), 2.0)):
        cut = sum(w for i, j, w in tri if bits[i] != bits[j])
        assert cut == want
    w = [(0, 1, 2.0), (1, 2, 3.0)]
    assert sum(x for i, j, x in w if (1, 0, 1)[i] != (1, 0, 1)[j]) == 5.0
    del probs


def test_qaoa_reference_runs():
    for n, edges, p, iters in ((3, [(0, 1, 1.0), (1, 2, 1.0), (0, 2, 1.0)], 2, 20),
                               (2, [(0, 1, 1.0)], 1, 20),
                               (4, [(0, 1, 1.0), (1, 2, 1.0), (2, 3, 1.0), (0, 3, 1.0)], 2, 30),
                               (4, [(0, 1, 1.0), (0, 2, 1.0), (0, 3, 1.0)], 2, 30)):
        r = oracle.run_qaoa(n, edges, p, iters, 0.1)
        assert r["best_cut_value"] >= 0.0          # test_algorithms.rs:466-545
        assert len(r["gammas"]) == p and len(r["betas"]) == p
        assert 0 <= r["best_bits"] < (1 << n)


def _h2():
    coeffs = [-1.0523, 0.3979, -0.3979, -0.0112, 0.1809]
    terms = [[], [(1, 3)], [(0, 3)], [(0, 3), (1, 3)], [(0, 1), (1, 1)]]
    return coeffs, terms


def test_vqe_h2_reference():
    c, t = _h2()
    r = oracle.run_vqe(2, 2, c, t, 50, 0.01, 0.1)
    assert r["best_energy"] < -0.8                 # test_algorithms.rs:329-346
    r = oracle.run_vqe(2, 2, c, t, 20, 0.001, 0.1)
    assert r["history"][-1] <= r["history"][0] + 1e-6   # test_algorithms.rs:412-434


def test_vqe_single_z_bounded():
    r = oracle.run_vqe(1, 1, [1.0], [[(0, 3)]], 30, 0.01, 0.1)
    assert math.isfinite(r["best_energy"]) and -1 - 1e-6 <= r["best_energy"] <= 1 + 1e-6   # :349-391
