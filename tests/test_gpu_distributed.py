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
