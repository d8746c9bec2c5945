"""rq_state_apply_kraus (one quantum-trajectory step of a single-qubit Kraus channel,
the sets of crates/ruqu-core/src/noise.rs:166-280) on the GPU vs the oracle.

Same amplitudes, same seed: every step must pick the same operator (the choice is an
integer decision on the shared uniform stream) and the amplitudes must agree to 1e-12
(complex f64) / 1e-5 (complex f32) max-abs, the operator probability to 1e-12 / 1e-6.
"""
import numpy as np
import pytest

import oracle
import ruqu_b200 as rq
from ruqu_b200 import Gate, QuantumState
from ruqu_b200.noise import (amplitude_damping_kraus, depolarizing_kraus, phase_damping_kraus,
                             thermal_relaxation_kraus)

pytestmark = pytest.mark.gpu

PREC = {"f64": oracle.RQ_F64, "f32": oracle.RQ_F32}
TOL = {"f64": 1e-12, "f32": 1e-5}
PTOL = {"f64": 1e-12, "f32": 1e-6}
H, X, RY, CNOT = 0, 1, 9, 12


def _random_state(n, seed):
    r = np.random.default_rng(seed)
    a = r.normal(size=1 << n) + 1j * r.normal(size=1 << n)
    return a / np.linalg.norm(a)


def _channels():
    return [depolarizing_kraus(0.2), amplitude_damping_kraus(0.35), phase_damping_kraus(0.5),
            thermal_relaxation_kraus(40.0, 25.0, 6.0)]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n", [4, 12, 20])
def test_kraus_trajectory_matches_oracle(prec, n):
    seed = 77 + n
    a = _random_state(n, n)
    g = QuantumState.from_amplitudes(a, n, prec, seed)
    o = oracle.OracleState.from_amplitudes(a, n, PREC[prec], seed)
    r = np.random.default_rng(5)
    chans = _channels()
    picks = []
    for step in range(24):
        q = int(r.integers(n))
        ops = chans[step % len(chans)]
        kg, pg = g.apply_kraus(q, ops)
        ko, po = o.apply_kraus(q, ops)
        assert kg == ko, (step, q)
        assert abs(pg - po) < PTOL[prec], (step, pg, po)
        picks.append(kg)
        if step % 4 == 3:   # gates between channel steps; both sides apply the same list
            gl = [(H, q, 0, 0.0), (RY, (q + 1) % n, 0, 0.3 * step), (CNOT, q, (q + 1) % n, 0.0)]
            _apply(g, gl)
            o.apply(gl)
        d = float(np.abs(g.state_vector() - o.amplitudes()).max())
        assert d < TOL[prec], (step, d)
    assert len(set(picks)) > 1       # the trajectory used more than one operator


def _apply(g, gl):
    make = {H: lambda q0, q1, a: Gate.H(q0), RY: lambda q0, q1, a: Gate.Ry(q0, a),
            CNOT: lambda q0, q1, a: Gate.CNOT(q0, q1)}
    g.apply_gates([make[k](q0, q1, a) for k, q0, q1, a in gl])


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_kraus_then_measure_shares_the_stream(prec):
    n, seed = 10, 3
    a = _random_state(n, 1)
    g = QuantumState.from_amplitudes(a, n, prec, seed)
    o = oracle.OracleState.from_amplitudes(a, n, PREC[prec], seed)
    for q in range(n):
        assert g.apply_kraus(q, amplitude_damping_kraus(0.3))[0] == o.apply_kraus(q, amplitude_damping_kraus(0.3))[0]
        m = g.measure((q + 3) % n)
        mo = o.measure((q + 3) % n)
        assert m.result == mo[1]
    assert float(np.abs(g.state_vector() - o.amplitudes()).max()) < TOL[prec]


def test_kraus_gamma1_resets_qubit():
    g = QuantumState(8, 0, "f64")
    _apply(g, [(H, 2, 0, 0.0)])
    g.apply_kraus(2, amplitude_damping_kraus(1.0))
    want = np.zeros(256, complex)
    want[0] = 1
    assert float(np.abs(g.state_vector() - want).max()) < 1e-15


def test_kraus_errors():
    g = QuantumState(4, 0, "f64")
    with pytest.raises(rq.InvalidQubitIndex):
        g.apply_kraus(4, depolarizing_kraus(0.1))
    with pytest.raises(rq.InvalidArgument):
        g.apply_kraus(0, np.zeros((0, 2, 2)))
    with pytest.raises(rq.InvalidArgument):
        g.apply_kraus(0, np.tile(np.eye(2) / 17 ** 0.5, (17, 1, 1)))
    with pytest.raises(rq.InvalidStateVector):
        g.apply_kraus(0, np.zeros((2, 2, 2)))
    # the failed calls left the state and its stream untouched
    assert float(np.abs(g.state_vector()[0] - 1)) < 1e-15
