"""Kraus channel sets (crates/ruqu-core/src/noise.rs:151-280) and the oracle's
trajectory step, on the CPU.

The first group restates the reference's own unit tests of the sets
(noise.rs:643-830): trace preservation at its parameter lists and tolerances, the
p=0 / lambda=0 / gate_time=0 identities and the gamma=1 decay of |1> to |0>.  The
second checks the oracle's ``apply_kraus`` (the checker of ``rq_state_apply_kraus``)
against numpy: the operator probabilities tr(K rho K^dagger) of the reduced density
matrix, the renormalised post-state, the draw it consumes, and that the average of
|psi><psi| over trajectories converges to the channel's output sum_k K rho K^dagger.
"""
import numpy as np
import pytest

import oracle
from ruqu_b200.noise import (amplitude_damping_kraus, completeness_error, depolarizing_kraus,
                             phase_damping_kraus, thermal_relaxation_kraus)


@pytest.mark.parametrize("p", [0.0, 0.01, 0.1, 0.5, 1.0])
def test_depolarizing_trace_preserving(p):
    assert completeness_error(depolarizing_kraus(p)) < 1e-12


def test_depolarizing_p0_is_identity():
    ops = depolarizing_kraus(0.0)
    assert ops.shape == (4, 2, 2)
    assert abs(ops[0, 0, 0] - 1) < 1e-14 and abs(ops[0, 1, 1] - 1) < 1e-14
    assert abs(ops[0, 0, 1]) ** 2 < 1e-28 and abs(ops[0, 1, 0]) ** 2 < 1e-28
    assert np.all(np.abs(ops[1:]) ** 2 < 1e-28)


@pytest.mark.parametrize("gamma", [0.0, 0.01, 0.1, 0.5, 0.99, 1.0])
def test_amplitude_damping_trace_preserving(gamma):
    assert completeness_error(amplitude_damping_kraus(gamma)) < 1e-12


def test_amplitude_damping_gamma1_decays_one_to_zero():
    ops = amplitude_damping_kraus(1.0)
    assert ops.shape == (2, 2, 2)
    assert abs(ops[0, 0, 0] - 1) < 1e-14 and abs(ops[0, 1, 1]) ** 2 < 1e-28
    assert abs(ops[1, 0, 1] - 1) < 1e-14 and abs(ops[1, 1, 0]) ** 2 < 1e-28 and abs(ops[1, 1, 1]) ** 2 < 1e-28
    out = ops[1] @ np.array([0, 1], dtype=complex)
    assert abs(out[0] - 1) < 1e-14 and abs(out[1]) ** 2 < 1e-28


@pytest.mark.parametrize("lam", [0.0, 0.01, 0.1, 0.5, 1.0])
def test_phase_damping_trace_preserving(lam):
    assert completeness_error(phase_damping_kraus(lam)) < 1e-12


def test_phase_damping_lambda0_is_identity():
    ops = phase_damping_kraus(0.0)
    assert ops.shape == (2, 2, 2)
    assert abs(ops[0, 0, 0] - 1) < 1e-14 and abs(ops[0, 1, 1] - 1) < 1e-14
    assert np.all(np.abs(ops[1]) ** 2 < 1e-28)


@pytest.mark.parametrize("t1,t2,gt", [(50.0, 30.0, 0.05), (50.0, 50.0, 0.05), (50.0, 100.0, 0.05),
                                      (100.0, 80.0, 1.0), (50.0, 30.0, 0.001)])
def test_thermal_relaxation_trace_preserving(t1, t2, gt):
    ops = thermal_relaxation_kraus(t1, t2, gt)
    assert ops.shape == (4, 2, 2)
    assert completeness_error(ops) < 1e-10


def test_thermal_relaxation_zero_gate_time_is_identity():
    ops = thermal_relaxation_kraus(50.0, 30.0, 0.0)
    assert ops.shape == (1, 2, 2)
    assert abs(ops[0, 0, 0] - 1) < 1e-14 and abs(ops[0, 1, 1] - 1) < 1e-14


def test_thermal_relaxation_order_is_ad_times_pd():
    t1, t2, gt = 50.0, 30.0, 0.5
    ops = thermal_relaxation_kraus(t1, t2, gt)
    gamma = 1 - np.exp(-gt / t1)
    lam = 1 - np.exp(-gt * (1 / t2 - 1 / (2 * t1)))
    ad, pd = amplitude_damping_kraus(gamma), phase_damping_kraus(lam)
    for i, (a, b) in enumerate([(a, b) for a in ad for b in pd]):
        np.testing.assert_allclose(ops[i], a @ b, rtol=0, atol=1e-15)


# ----------------------------------------------------------------- oracle trajectory step
def _random_state(n, seed):
    r = np.random.default_rng(seed)
    a = r.normal(size=1 << n) + 1j * r.normal(size=1 << n)
    return a / np.linalg.norm(a)


def _reduced(a, n, q):
    t = a.reshape([2] * n)              # axis j holds bit n-1-j
    ax = n - 1 - q
    t = np.moveaxis(t, ax, 0).reshape(2, -1)
    return t @ t.conj().T               # rho_ij = sum a_i conj(a_j)


def _apply_1q(a, n, q, m):
    t = np.moveaxis(a.reshape([2] * n), n - 1 - q, 0)
    t = np.tensordot(m, t, axes=(1, 0))
    return np.moveaxis(t, 0, n - 1 - q).reshape(-1)


CHANNELS = {
    "depolarizing": depolarizing_kraus(0.3),
    "amplitude_damping": amplitude_damping_kraus(0.4),
    "phase_damping": phase_damping_kraus(0.25),
    "thermal": thermal_relaxation_kraus(50.0, 30.0, 5.0),
}


@pytest.mark.parametrize("name", sorted(CHANNELS))
@pytest.mark.parametrize("q", [0, 3, 5])
def test_oracle_kraus_step_matches_numpy(name, q):
    n, seed = 6, 11
    ops = CHANNELS[name]
    a = _random_state(n, 3 + q)
    st = oracle.OracleState.from_amplitudes(a, n, oracle.RQ_F64, seed)
    rho = _reduced(a, n, q)
    pk = np.array([np.trace(k @ rho @ k.conj().T).real for k in ops])
    u = oracle.uniform(seed, 0, 0)      # the first draw of the state's stream
    want = int(np.searchsorted(np.cumsum(pk / pk.sum()), u, side="right"))
    k, p = st.apply_kraus(q, ops)
    assert k == want
    assert abs(p - pk[k] / pk.sum()) < 1e-13
    post = _apply_1q(a, n, q, ops[k]) / np.sqrt(pk[k])
    assert np.abs(st.amplitudes() - post).max() < 1e-13
    assert abs(np.linalg.norm(st.amplitudes()) - 1) < 1e-13


def test_oracle_kraus_draws_follow_the_measurement_stream():
    """A Kraus step takes exactly one draw: a measurement after it uses draw 1."""
    n, seed = 4, 5
    a = _random_state(n, 9)
    st = oracle.OracleState.from_amplitudes(a, n, oracle.RQ_F64, seed)
    st.apply_kraus(1, depolarizing_kraus(0.0))      # K0 = I: probability 1, state unchanged
    assert np.abs(st.amplitudes() - a).max() < 1e-15
    res = st.measure(2)
    p0 = float(np.sum(np.abs(a[(np.arange(1 << n) >> 2) & 1 == 0]) ** 2))
    assert res[1] == (oracle.uniform(seed, 0, 1) >= p0)


def test_oracle_amplitude_damping_gamma1_resets_to_zero():
    n = 3
    st = oracle.OracleState(n, oracle.RQ_F64, 1)
    st.apply([(1, 1, 0, 0.0)])                      # X on qubit 1
    k, p = st.apply_kraus(1, amplitude_damping_kraus(1.0))
    assert (k, p) == (1, 1.0)
    want = np.zeros(1 << n, complex)
    want[0] = 1
    assert np.abs(st.amplitudes() - want).max() < 1e-15


def test_oracle_trajectories_average_to_the_channel():
    n, q, shots = 3, 1, 3000
    ops = thermal_relaxation_kraus(20.0, 15.0, 8.0)
    a = _random_state(n, 21)
    rho_full = np.outer(a, a.conj())
    # the channel on the full density matrix: sum_k (K_k)_q rho (K_k)_q^dagger
    want = np.zeros((1 << n, 1 << n), complex)
    for k in ops:
        kf = np.array([_apply_1q(col, n, q, k) for col in np.eye(1 << n)]).T
        want += kf @ rho_full @ kf.conj().T
    acc = np.zeros_like(want)
    for s in range(shots):
        st = oracle.OracleState.from_amplitudes(a, n, oracle.RQ_F64, 1000 + s)
        st.apply_kraus(q, ops)
        b = st.amplitudes()
        acc += np.outer(b, b.conj())
    err = np.abs(acc / shots - want).max()
    assert err < 4.0 / np.sqrt(shots), err


def test_oracle_kraus_errors():
    st = oracle.OracleState(2, oracle.RQ_F64, 0)
    with pytest.raises(oracle.OracleError):
        st.apply_kraus(2, depolarizing_kraus(0.1))
    with pytest.raises(oracle.OracleError):
        st.apply_kraus(0, np.zeros((1, 2, 2)))      # annihilates the state
