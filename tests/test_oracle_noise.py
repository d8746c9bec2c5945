"""The oracle's noise loop (Simulator::run_with_config with a NoiseModel,
simulator.rs:67-78 and apply_noise, simulator.rs:177-221) against a second,
independent restatement of the draw order written here in Python.

The reference draws from the state's ChaCha12 generator; here both sides draw
from the documented Philox uniform stream, the same one measurements use
(RNG draws are unpinned; what is pinned is the order and the decisions).
"""
import numpy as np
import pytest

import oracle
from ruqu_b200 import workloads

H, X, Y, Z, CNOT, CZ, SWAP, RZZ, MEASURE, RESET, BARRIER = 0, 1, 2, 3, 12, 13, 14, 15, 16, 17, 18
TWO_Q = (CNOT, CZ, SWAP, RZZ)


def expand(gates, seed, rates, start=0):
    """The list with apply_noise's Paulis inserted after their gates, for lists
    without Measure / Reset; returns (list, draws consumed)."""
    dep, bf, pf = rates
    d = start
    out = []
    for g in gates:
        out.append(g)
        if g[0] == BARRIER:
            continue
        for q in ([g[1], g[2]] if g[0] in TWO_Q else [g[1]]):
            if dep > 0:
                r = oracle.uniform(seed, 0, d)
                d += 1
                if r < dep:
                    c = oracle.uniform(seed, 0, d)
                    d += 1
                    out.append((X if c < 1 / 3 else (Y if c < 2 / 3 else Z), q, 0, 0.0))
            if bf > 0:
                r = oracle.uniform(seed, 0, d)
                d += 1
                if r < bf:
                    out.append((X, q, 0, 0.0))
            if pf > 0:
                r = oracle.uniform(seed, 0, d)
                d += 1
                if r < pf:
                    out.append((Z, q, 0, 0.0))
    return out, d


@pytest.mark.parametrize("rates", [(0.1, 0.05, 0.07), (0.3, 0.0, 0.0), (0.0, 0.2, 0.0), (0.0, 0.0, 0.25)])
def test_noise_loop_matches_the_draw_order(rates):
    n, seed = 8, 11
    gates = workloads.random_layer_circuit(n, 3, 5)
    gates.insert(20, (BARRIER, 0, 0, 0.0))
    gates.append((RZZ, 2, 5, 0.7))
    noisy = oracle.OracleState(n, seed=seed)
    noisy.apply_noisy(gates, rates)
    ex, _ = expand(gates, seed, rates)
    assert len(ex) > len(gates)                    # some noise fired
    ref = oracle.OracleState(n, seed=seed)
    ref.apply(ex)
    assert np.array_equal(noisy.amplitudes(), ref.amplitudes())


def test_depolarising_picks_all_three_paulis():
    gates = workloads.random_layer_circuit(8, 4, 6)
    ex, _ = expand(gates, 3, (0.5, 0.0, 0.0))
    assert {g[0] for g in ex if g[0] in (X, Y, Z)} == {X, Y, Z}   # the circuit itself has none


def test_zero_rates_draw_nothing():
    n, seed = 6, 4
    gates = workloads.random_layer_circuit(n, 2, 2)
    a = oracle.OracleState(n, seed=seed)
    a.apply_noisy(gates, (0.0, 0.0, 0.0))
    b = oracle.OracleState(n, seed=seed)
    b.apply(gates)
    assert np.array_equal(a.amplitudes(), b.amplitudes())
    # the measurement stream is where it was: the next measurements agree
    ma = [a.measure(q) for q in range(n)]
    mb = [b.measure(q) for q in range(n)]
    assert ma == mb


@pytest.mark.parametrize("seed", [1, 2, 3, 4, 5, 6, 7, 8])
def test_measurement_keeps_its_place_in_the_stream(seed):
    """H(0); Measure(0) with bit flips certain: draw 0 flips after H, draw 1 is the
    measurement's (|+> stays |+> under X, p0 = 1/2), draw 2 flips after Measure."""
    s = oracle.OracleState(1, seed=seed)
    rec = s.apply_noisy([(H, 0, 0, 0.0), (MEASURE, 0, 0, 0.0)], (0.0, 1.0, 0.0))
    want = oracle.uniform(seed, 0, 1) >= 0.5
    assert rec[0][1] == want
    # after the post-measurement flip the qubit holds the opposite value
    amps = s.amplitudes()
    assert abs(abs(amps[0 if want else 1]) - 1.0) < 1e-12
