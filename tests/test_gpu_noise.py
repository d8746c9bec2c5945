"""Noisy runs on the device (rq_state_apply_noisy) vs the oracle's restatement of
Simulator::run_with_config with a NoiseModel (simulator.rs:67-78, 177-221) on the
same seed and uniform stream (needs a GPU).

Measurement records must agree exactly (outcomes); probabilities and amplitudes
to 1e-12 for f64 states (per-gate kernels at < 12 qubits, sweeps above).  For f32
states amplitudes agree to 1e-5 and probabilities to 2e-4: the reference sums p0
sequentially in f32 (mixed_precision.rs:480), whose rounding grows with 2^n
(about sqrt(2^n) * 2^-24 typically, 2^n * 2^-24 at worst: 1.5e-5 / 3.9e-3 at 16 qubits).
"""
import numpy as np
import pytest

import oracle
import ruqu_b200 as rq
from ruqu_b200 import workloads

pytestmark = pytest.mark.gpu

H, X, Y, Z, CNOT, MEASURE, RESET, BARRIER = 0, 1, 2, 3, 12, 16, 17, 18


def _circuit(n, layers, seed):
    g = workloads.random_layer_circuit(n, layers, seed)
    k = len(g) // 3
    # mid-circuit measurement, reset and barrier (noise also follows Measure and Reset)
    return g[:k] + [(MEASURE, 1, 0, 0.0), (BARRIER, 0, 0, 0.0), (RESET, 2, 0, 0.0)] + g[k:] + [(MEASURE, 0, 0, 0.0)]


def _compare(n, gates, rates, seed, prec, tol):
    s = rq.QuantumState(n, seed, prec)
    rec = s.apply_gates_noisy(gates, rq.NoiseModel(*rates))
    o = oracle.OracleState(n, oracle.RQ_F64 if prec == "f64" else oracle.RQ_F32, seed=seed)
    orec = o.apply_noisy(gates, rates)
    assert [(m.qubit, m.result) for m in rec] == [(q, r) for q, r, _ in orec]
    ptol = tol if prec == "f64" else 2e-4
    dp = max((abs(m.probability - p) for m, (_, _, p) in zip(rec, orec)), default=0.0)
    assert dp < ptol, dp
    assert np.max(np.abs(s.state_vector() - o.amplitudes())) < tol
    # the stream continues where the noisy run left it
    assert [s.measure(q).result for q in range(3)] == [o.measure(q)[1] for q in range(3)]


@pytest.mark.parametrize("seed", [3, 9])
def test_noisy_run_f64_per_gate(seed):
    _compare(10, _circuit(10, 4, seed), (0.05, 0.02, 0.03), seed, "f64", 1e-12)


def test_noisy_run_f64_sweeps():
    _compare(14, _circuit(14, 4, 2), (0.04, 0.03, 0.02), 5, "f64", 1e-12)


def test_noisy_run_f32_sweeps():
    _compare(16, _circuit(16, 3, 4), (0.05, 0.0, 0.05), 8, "f32", 1e-5)


def test_zero_rates_equal_the_plain_run():
    n, seed = 12, 6
    gates = _circuit(n, 3, 1)
    a = rq.QuantumState(n, seed, "f64")
    ra = a.apply_gates_noisy(gates, rq.NoiseModel())
    b = rq.QuantumState(n, seed, "f64")
    rb = b.apply_gates(gates)
    assert ra == rb
    assert np.array_equal(a.state_vector(), b.state_vector())


def test_simulator_run_with_config_takes_the_noise_model():
    n = 9
    c = rq.QuantumCircuit(n)
    for q in range(n):
        c.h(q)
    for q in range(n - 1):
        c.cnot(q, q + 1)
    c.measure(4)
    noise = rq.NoiseModel(depolarizing_rate=0.1, bit_flip_rate=0.05, phase_flip_rate=0.05)
    r = rq.Simulator.run_with_config(c, rq.SimConfig(seed=17, noise=noise))
    o = oracle.OracleState(n, seed=17)
    orec = o.apply_noisy([g.to_tuple() for g in c.gates()], (0.1, 0.05, 0.05))
    assert [(m.qubit, m.result) for m in r.measurements] == [(q, v) for q, v, _ in orec]
    assert np.max(np.abs(r.state.state_vector() - o.amplitudes())) < 1e-12
