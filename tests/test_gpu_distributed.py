"""A distributed state on the device (needs a GPU): all 2^g ranks' local states live
on one GPU (StateGroup of DeviceRank states), so the pack / unpack kernels
(rq_state_half_copy), the per-rank translation and the local sweeps all run on the
device; the result must match one QuantumState of all n qubits running the same
gates: 1e-12 for f64 states, 1e-5 for f32 states (amplitudes and expectations).
Only one GPU is used: the ranks' exchanges are buffer swaps, not NCCL transfers.
"""
import math

import numpy as np
import pytest

import ruqu_b200 as rq
from ruqu_b200 import workloads
from ruqu_b200.distributed import DeviceRank, StateGroup

pytestmark = pytest.mark.gpu

H, X, Y, Z, S, SDG, T, TDG, RX, RY, RZ, PHASE, CNOT, CZ, SWAP, RZZ = range(16)


def _random_circuit(n, count, seed):
    rng = np.random.default_rng(seed)
    kinds1 = [H, X, Y, Z, S, SDG, T, TDG, RX, RY, RZ, PHASE]
    out = []
    for _ in range(count):
        if rng.random() < 0.6:
            out.append((int(rng.choice(kinds1)), int(rng.integers(n)), 0, float(rng.uniform(0, 2 * math.pi))))
        else:
            a, b = rng.choice(n, size=2, replace=False)
            out.append((int(rng.choice([CNOT, CZ, SWAP, RZZ])), int(a), int(b), float(rng.uniform(0, 2 * math.pi))))
    return out


def _strings(n, seed):
    rng = np.random.default_rng(seed)
    out = [[(q, 3)] for q in range(n)]
    for _ in range(10):
        qs = rng.choice(n, size=4, replace=False)
        out.append([(int(q), int(rng.integers(1, 4))) for q in qs])
    return out


@pytest.mark.parametrize("n,g,prec,seed", [(12, 1, "f64", 1), (14, 2, "f64", 2), (13, 3, "f64", 3),
                                           (16, 2, "f32", 4)])
def test_group_on_device_matches_one_state(n, g, prec, seed):
    gates = _random_circuit(n, 200, seed)
    grp = StateGroup(n, g, prec, engines=[DeviceRank(n - g, 0, prec) for _ in range(1 << g)])
    grp.apply_gates(gates)
    one = rq.QuantumState(n, 0, prec)
    one.apply_gates(gates)
    tol = 1e-12 if prec == "f64" else 1e-5
    assert np.max(np.abs(grp.state_vector() - one.state_vector())) < tol
    st = _strings(n, seed + 10)
    assert np.max(np.abs(grp.expectation_values(st) - one.expectation_values(st))) < tol


def test_random_layers_20_qubits_over_four_ranks_f32():
    """The benchmark's circuit family at 20 qubits: 18 local qubits per rank, so the local
    runs go through the sweep path."""
    n, g = 20, 2
    gates = workloads.random_layer_circuit(n, 6, 1)
    grp = StateGroup(n, g, "f32", engines=[DeviceRank(n - g, 0, "f32") for _ in range(1 << g)])
    grp.apply_gates(gates)
    one = rq.QuantumState(n, 0, "f32")
    one.apply_gates(gates)
    assert np.max(np.abs(grp.state_vector() - one.state_vector())) < 1e-5
    z = [[(q, 3)] for q in range(n)]
    assert np.max(np.abs(grp.expectation_values(z) - one.expectation_values(z))) < 1e-5


def test_half_copy_round_trip():
    import torch
    s = rq.QuantumState(10, 0, "f64")
    r = np.random.default_rng(5)
    a = r.normal(size=1024) + 1j * r.normal(size=1024)
    s.set_amplitudes(a)
    buf = torch.empty(512 * 16, dtype=torch.uint8, device="cuda")
    s.half_copy(3, 1, buf.data_ptr())
    s.synchronize()
    got = buf.cpu().numpy().view(np.complex128)
    i = np.arange(1024)
    assert np.array_equal(got, a[((i >> 3) & 1) == 1])
    buf2 = torch.from_numpy(np.ascontiguousarray(np.conj(got)).view(np.uint8)).cuda()
    torch.cuda.synchronize()
    s.half_copy(3, 1, buf2.data_ptr(), unpack=True)
    want = a.copy()
    want[((i >> 3) & 1) == 1] = np.conj(got)
    assert np.array_equal(s.state_vector(), want)
    with pytest.raises(rq.InvalidArgument):
        s.half_copy(3, 2, buf.data_ptr())


def test_prefix_tree_lookups_match_numpy():
    """rq_state_tree_build / rq_state_tree_lookup: level L, entry j = sum of |a|^2 over the
    amplitudes whose first L tree qubits (the listed order, then the rest) take the bits of
    j; level 0 is the squared norm, level n the probabilities."""
    n = 11
    r = np.random.default_rng(3)
    a = r.normal(size=1 << n) + 1j * r.normal(size=1 << n)
    for prec, tol in (("f64", 1e-12), ("f32", 1e-6)):
        s = rq.QuantumState.from_amplitudes(a, n, prec)
        with pytest.raises(rq.InvalidArgument):
            s.tree_lookup(0, [0])                      # no tree yet
        amps = s.state_vector()
        p = np.abs(amps) ** 2
        for listed in ([3, 0, 7], [10, 2, 2, 5, 1], []):
            s.tree_build(listed)
            order = list(dict.fromkeys(listed)) + [q for q in range(n) if q not in listed]
            j = np.arange(1 << n)
            src = np.zeros_like(j)
            for k, q in enumerate(order):
                src |= ((j >> k) & 1) << q
            pj = p[src]
            for level in range(n + 1):
                want = pj.reshape(-1, 1 << level).sum(axis=0)
                idx = np.arange(1 << level, dtype=np.uint64)
                got = s.tree_lookup(level, idx)
                assert np.max(np.abs(got - want)) < tol * max(1.0, float(np.sum(p))), (prec, listed, level)
        with pytest.raises(rq.InvalidArgument):
            s.tree_lookup(3, [8])
        with pytest.raises(rq.InvalidArgument):
            s.tree_lookup(n + 1, [0])
        with pytest.raises(rq.InvalidQubitIndex):
            s.tree_build([n])


@pytest.mark.parametrize("n,g,prec,seed", [(12, 1, "f64", 5), (13, 2, "f64", 6), (14, 2, "f32", 7)])
def test_group_measure_reset_sample_on_device_match_one_state(n, g, prec, seed):
    """measure / reset_qubit / Measure gates / sample of a distributed state (all ranks on
    this GPU) equal one QuantumState's with the same measurement seed: outcomes and shots
    exact, probabilities and amplitudes 1e-12 (f64) / 1e-5 (f32)."""
    tol = 1e-12 if prec == "f64" else 1e-5
    gates = _random_circuit(n, 150, seed)
    grp = StateGroup(n, g, prec, seed=seed, engines=[DeviceRank(n - g, 0, prec) for _ in range(1 << g)])
    one = rq.QuantumState(n, seed, prec)
    grp.apply_gates(gates)
    one.apply_gates(gates)
    glob = next(q for q in range(n) if not grp.layout.is_local(q))
    loc = next(q for q in range(n) if grp.layout.is_local(q))
    for q in (glob, loc, glob):
        a, b = grp.measure(q), one.measure(q)
        assert (a.qubit, a.result) == (b.qubit, b.result)
        assert abs(a.probability - b.probability) < tol
        assert np.max(np.abs(grp.state_vector() - one.state_vector())) < tol
    more = _random_circuit(n, 60, seed + 1) + [(16, loc, 0, 0.0), (17, glob, 0, 0.0)]
    got = grp.apply_gates(more)
    want = one.apply_gates(more)
    assert [(o.qubit, o.result) for o in got] == [(o.qubit, o.result) for o in want]
    assert np.max(np.abs(grp.state_vector() - one.state_vector())) < tol
    grp.apply_gates([(H, k, 0, 0.0) for k in range(0, n, 2)])
    one.apply_gates([(H, k, 0, 0.0) for k in range(0, n, 2)])
    for qubits in (None, [glob, loc, 3, glob]):
        assert np.array_equal(grp.sample(1024, 42, qubits), one.sample(1024, 42, qubits)), qubits
