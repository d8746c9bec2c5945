"""Grover search with the amplitude edits on the device vs the reference's host-edit
loop restated on the oracle state (grover.rs:99-184), and the reference's Grover
tests (test_algorithms.rs:180-318) (needs a GPU).

Negations are exact, so amplitudes agree to the Hadamard layers' rounding
(1e-12, f64); the measured state and the success probability agree because both
sides draw the measurements from the same seeded stream.
"""
import numpy as np
import pytest

import oracle
import ruqu_b200 as rq
from ruqu_b200.grover import GroverConfig, optimal_iterations, run_grover

pytestmark = pytest.mark.gpu

H, MEASURE = 0, 16


def _oracle_grover(n, targets, iterations, seed):
    o = oracle.OracleState(n, seed=seed)
    hs = [(H, q, 0, 0.0) for q in range(n)]
    o.apply(hs)
    for _ in range(iterations):
        a = o.amplitudes()
        for t in targets:            # grover.rs:130-139, one negation per listed target
            a[t] = -a[t]
        o.upload(a)
        o.apply(hs)
        a = o.amplitudes()
        a[1:] = -a[1:]               # grover.rs:145-153
        o.upload(a)
        o.apply(hs)
    p = o.probabilities()
    success = float(sum(p[t] for t in targets))
    measured = 0
    for q in range(n):
        if o.measure(q)[1]:
            measured |= 1 << q
    return o, success, measured


@pytest.mark.parametrize("n,targets,seed", [(4, [7], 42), (3, [5], 42), (3, [0], 42), (3, [1, 5], 123),
                                            (3, [0, 2, 4, 6], 42), (10, [3, 700], 5), (13, [4097], 9),
                                            (6, [9, 9, 12], 2)])
def test_grover_matches_the_host_edit_loop(n, targets, seed):
    r = run_grover(GroverConfig(n, targets, None, seed))
    k = optimal_iterations(n, len(targets))
    o, success, measured = _oracle_grover(n, targets, k, seed)
    assert r.num_iterations == k
    assert abs(r.success_probability - success) < 1e-12
    assert r.measured_state == measured
    assert r.target_found == (measured in targets)
    assert np.max(np.abs(r.state.state_vector() - o.amplitudes())) < 1e-12


def test_reference_grover_thresholds():
    """test_algorithms.rs:180-318."""
    assert run_grover(GroverConfig(4, [7], None, 42)).success_probability > 0.8
    assert run_grover(GroverConfig(3, [5], None, 42)).success_probability > 0.8
    assert run_grover(GroverConfig(3, [0], None, 42)).success_probability > 0.8
    assert run_grover(GroverConfig(3, [1, 5], None, 123)).success_probability > 0.7
    assert run_grover(GroverConfig(3, [0, 2, 4, 6], None, 42)).success_probability > 0.5
    assert run_grover(GroverConfig(3, [3], 2, 42)).num_iterations == 2
    assert run_grover(GroverConfig(3, [6], None, 42)).measured_state < 8


def test_negate_ops_on_the_device():
    n = 5
    r = np.random.default_rng(3)
    a = r.normal(size=1 << n) + 1j * r.normal(size=1 << n)
    s = rq.QuantumState(n, 0, "f64")
    s.set_amplitudes(a)
    s.negate_amplitudes([3, 7, 7, 31, 3, 3])      # 3 three times, 7 twice, 31 once
    want = a.copy()
    want[[3, 31]] *= -1
    assert np.array_equal(s.state_vector(), want)
    s.negate_all_except(4)
    want = -want
    want[4] = -want[4]
    assert np.array_equal(s.state_vector(), want)
    with pytest.raises(rq.InvalidArgument):
        s.negate_amplitudes([1, 32])                # out of range: nothing changes
    assert np.array_equal(s.state_vector(), want)
    s.negate_amplitudes([])
    assert np.array_equal(s.state_vector(), want)
