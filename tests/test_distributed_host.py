"""The distributed state's schedule, per-rank translation and exchanges on the CPU
(ruqu_b200/distributed.py): every rank's local state is an oracle state, so what is
checked is the distribution logic itself against one oracle state of all n qubits.

* StateGroup (all ranks in this process) on random circuits with every gate kind;
* DistributedState over gloo with 2 and 4 processes (the SPMD path: send / receive
  of the packed halves between ranks);
* the schedule: diagonal gates on global qubits need no exchange, SWAP only relabels.
Amplitudes agree to 1e-12, expectations to 1e-12.
"""
import math
import os
import socket

import numpy as np
import pytest
import torch

import oracle
from ruqu_b200.distributed import Layout, StateGroup, schedule

H, X, Y, Z, S, SDG, T, TDG, RX, RY, RZ, PHASE, CNOT, CZ, SWAP, RZZ, MEASURE, RESET, BARRIER, U1 = range(20)


class OracleRank:
    """A rank's local state held by the oracle (test stand-in for the device state)."""

    def __init__(self, nl):
        self.nl = nl
        self.s = oracle.OracleState(nl, seed=0)

    def _idx(self, p, v):
        i = np.arange(1 << self.nl)
        return i[((i >> p) & 1) == v]

    def apply(self, gates):
        if gates:
            self.s.apply(gates)

    def zero(self):
        self.s.upload(np.zeros(1 << self.nl, dtype=np.complex128))

    def pack(self, p, v):
        a = self.s.amplitudes()[self._idx(p, v)]
        return torch.from_numpy(np.ascontiguousarray(a).view(np.float64).copy())

    def recv_buffer(self):
        return torch.empty(1 << self.nl, dtype=torch.float64)

    def unpack(self, p, v, buf):
        a = self.s.amplitudes()
        a[self._idx(p, v)] = buf.numpy().view(np.complex128)
        self.s.upload(a)

    def expectation(self, strings):
        return [self.s.expectation(st) if st else float(np.sum(np.abs(self.s.amplitudes()) ** 2)) for st in strings]

    def tree_build(self, bits):
        """The sampler's prefix tree over the local bits in that order (the rest after them):
        entry j of level L sums |a|^2 over the amplitudes whose first L ordered bits are j."""
        p = np.abs(self.s.amplitudes()) ** 2
        order = list(bits) + [b for b in range(self.nl) if b not in bits]
        j = np.arange(1 << self.nl)
        src = np.zeros_like(j)
        for k, b in enumerate(order):
            src |= ((j >> k) & 1) << b
        self._pj = p[src]

    def tree_lookup(self, level, index):
        return self._pj.reshape(-1, 1 << level).sum(axis=0)[np.asarray(index, dtype=np.int64)]

    def amplitudes(self):
        return self.s.amplitudes()


def random_circuit(n, count, rng):
    kinds1 = [H, X, Y, Z, S, SDG, T, TDG, RX, RY, RZ, PHASE]
    out = []
    for _ in range(count):
        r = rng.random()
        if r < 0.55:
            out.append((int(rng.choice(kinds1)), int(rng.integers(n)), 0, float(rng.uniform(0, 2 * math.pi))))
        elif r < 0.6:
            m = np.linalg.qr(rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)))[0]
            out.append((U1, int(rng.integers(n)), 0, 0.0, [m[0, 0].real, m[0, 0].imag, m[0, 1].real, m[0, 1].imag,
                                                          m[1, 0].real, m[1, 0].imag, m[1, 1].real, m[1, 1].imag]))
        elif r < 0.62:
            out.append((BARRIER, 0, 0, 0.0))
        else:
            a, b = rng.choice(n, size=2, replace=False)
            out.append((int(rng.choice([CNOT, CZ, SWAP, RZZ])), int(a), int(b), float(rng.uniform(0, 2 * math.pi))))
    return out


def random_strings(n, count, rng, max_flips=4):
    out = []
    while len(out) < count:
        ops = rng.integers(0, 4, size=n)
        if np.sum((ops == 1) | (ops == 2)) > max_flips:
            continue
        out.append([(q, int(o)) for q, o in enumerate(ops) if o])
    out.append([])
    return out


def _full(n, gates):
    o = oracle.OracleState(n, seed=0)
    o.apply([g for g in gates if g[0] != BARRIER])
    return o


@pytest.mark.parametrize("n,g,seed", [(7, 1, 1), (8, 2, 2), (9, 3, 3), (10, 2, 4), (6, 1, 5)])
def test_group_matches_one_state(n, g, seed):
    rng = np.random.default_rng(seed)
    gates = random_circuit(n, 120, rng)
    grp = StateGroup(n, g, engines=[OracleRank(n - g) for _ in range(1 << g)])
    grp.apply_gates(gates)
    full = _full(n, gates)
    assert np.max(np.abs(grp.state_vector() - full.amplitudes())) < 1e-12
    strings = random_strings(n, 12, rng)
    want = [full.expectation(st) if st else 1.0 for st in strings]
    assert np.max(np.abs(grp.expectation_values(strings) - np.asarray(want))) < 1e-12
    # more gates after the expectation's exchanges (the layout moved on)
    more = random_circuit(n, 40, rng)
    grp.apply_gates(more)
    full.apply([x for x in more if x[0] != BARRIER])
    assert np.max(np.abs(grp.state_vector() - full.amplitudes())) < 1e-12


def test_diagonal_gates_on_global_qubits_need_no_exchange():
    lay = Layout(8, 2)
    gates = [(RZ, 7, 0, 0.3), (CZ, 6, 7, 0.0), (RZZ, 1, 7, 0.7), (CNOT, 6, 2, 0.0), (PHASE, 6, 0, 1.1), (T, 7, 0, 0.0)]
    steps = schedule(gates, lay)
    assert [s[0] for s in steps] == ["local"]
    assert lay.phys == list(range(8))


def test_swap_gate_only_relabels():
    lay = Layout(6, 2)
    steps = schedule([(SWAP, 0, 5, 0.0), (H, 0, 0, 0.0)], lay)
    assert [s[0] for s in steps] == ["swap", "local"]      # H on logical 0, now at a global bit
    lay2 = Layout(6, 2)
    steps2 = schedule([(SWAP, 0, 5, 0.0), (H, 5, 0, 0.0)], lay2)
    assert [s[0] for s in steps2] == ["local"]             # logical 5 sits on local bit 0


def test_furthest_next_use_is_given_up():
    lay = Layout(5, 1)     # local bits 0..3, qubit 4 global
    gates = [(H, 4, 0, 0.0), (H, 0, 0, 0.0), (H, 1, 0, 0.0), (H, 2, 0, 0.0)]
    steps = schedule(gates, lay)
    assert steps[0] == ("swap", 3, 0)                      # qubit 3 is never needed again
    assert lay.is_local(4) and not lay.is_local(3)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _spmd_worker(rank, world, port, n, seed, q):
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
        import datetime

        import torch.distributed as tdist

        from ruqu_b200.distributed import DistributedState
        tdist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        g = world.bit_length() - 1
        st = DistributedState(n, engine=OracleRank(n - g))
        rng = np.random.default_rng(seed)
        gates = random_circuit(n, 100, rng)
        st.apply_gates(gates)
        strings = random_strings(n, 8, rng)
        ev = st.expectation_values(strings)
        sv = st.state_vector()
        outs = [st.measure(x) for x in (n - 1, 0)]
        shots = st.sample(300, 5)
        sv2 = st.state_vector()
        tdist.barrier()
        tdist.destroy_process_group()
        if rank == 0:
            q.put(("ok", gates, strings, ev, sv, [(o.qubit, o.result, o.probability) for o in outs], shots, sv2))
    except Exception as e:     # report to the parent instead of hanging it
        q.put(("error", repr(e)))


@pytest.mark.parametrize("world,n", [(2, 7), (4, 8)])
def test_spmd_over_gloo_matches_one_state(world, n):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_spmd_worker, args=(r, world, port, n, 11, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
    assert res[0] == "ok", res
    _, gates, strings, ev, sv, outs, shots, sv2 = res
    full = _full(n, gates)
    assert np.max(np.abs(sv - full.amplitudes())) < 1e-12
    want = [full.expectation(st) if st else 1.0 for st in strings]
    assert np.max(np.abs(ev - np.asarray(want))) < 1e-12
    for (qb, r, pr), x in zip(outs, (n - 1, 0)):
        w = full.measure(x)
        assert (qb, r) == (w[0], w[1]) and abs(pr - w[2]) < 1e-12
    assert np.max(np.abs(sv2 - full.amplitudes())) < 1e-12
    want = oracle.tree_sample(np.abs(full.amplitudes()) ** 2, n, list(range(n)), 5, 300)
    assert np.array_equal(shots, want)


def _group(n, g, seed, gates):
    grp = StateGroup(n, g, seed=seed, engines=[OracleRank(n - g) for _ in range(1 << g)])
    full = oracle.OracleState(n, seed=seed)
    ops = [x for x in gates if x[0] != BARRIER]
    grp.apply_gates(ops)
    full.apply(ops)
    return grp, full


def _split(grp):
    """(a qubit held on a rank bit, a qubit held on a local bit) under the current layout."""
    glob = next(q for q in range(grp.n) if not grp.layout.is_local(q))
    loc = next(q for q in range(grp.n) if grp.layout.is_local(q))
    return glob, loc


@pytest.mark.parametrize("n,g,seed", [(7, 1, 1), (8, 2, 2), (9, 3, 3), (6, 2, 4)])
def test_group_measure_and_reset_match_one_state(n, g, seed):
    """measure / reset_qubit / measure_all / Measure and Reset gates of a distributed state
    equal QuantumState's (state.rs:288-352) on one oracle state with the same stream:
    outcomes exact, probabilities and amplitudes to 1e-12, on global and local qubits."""
    rng = np.random.default_rng(seed)
    grp, full = _group(n, g, seed, random_circuit(n, 80, rng))
    for _ in range(3):
        for q in _split(grp):
            out, want = grp.measure(q), full.measure(q)
            assert (out.qubit, out.result) == (want[0], want[1])
            assert abs(out.probability - want[2]) < 1e-12
            assert np.max(np.abs(grp.state_vector() - full.amplitudes())) < 1e-12
        more = [x for x in random_circuit(n, 30, rng) if x[0] != BARRIER]
        grp.apply_gates(more)
        full.apply(more)
    for q in _split(grp):
        grp.reset_qubit(q)
        full.reset_qubit(q)
        assert np.max(np.abs(grp.state_vector() - full.amplitudes())) < 1e-12
    tail = [(H, k, 0, 0.0) for k in range(n)] + [(MEASURE, n - 1, 0, 0.0), (RESET, 0, 0, 0.0), (CNOT, 0, n - 1, 0.0),
                                                  (MEASURE, 1, 0, 0.0)]
    got = grp.apply_gates(tail)
    want = full.apply(tail)
    assert [(o.qubit, o.result) for o in got] == [(w[0], w[1]) for w in want]
    assert np.max(np.abs(grp.state_vector() - full.amplitudes())) < 1e-12
    grp.apply_gates([(H, k, 0, 0.0) for k in range(n)])
    full.apply([(H, k, 0, 0.0) for k in range(n)])
    outs = grp.measure_all()
    want = [full.measure(q) for q in range(n)]
    assert [(o.qubit, o.result) for o in outs] == [(w[0], w[1]) for w in want]
    assert np.max(np.abs(grp.state_vector() - full.amplitudes())) < 1e-12
    assert len(grp.measurement_record) == 3 * 2 + 2 + 3 + n     # reset_qubit measures too


@pytest.mark.parametrize("n,g,seed", [(7, 1, 1), (8, 2, 2), (9, 3, 3)])
def test_group_sample_matches_the_tree_sampler(n, g, seed):
    """Shots of a distributed state equal the one-state sampler's (simulator.rs:107-147
    semantics) on the same probabilities: all qubits, a subset in a shuffled order with a
    repeat, and a single global qubit."""
    rng = np.random.default_rng(seed)
    grp, full = _group(n, g, seed, random_circuit(n, 100, rng))
    probs = np.abs(full.amplitudes()) ** 2
    glob, loc = _split(grp)
    for qubits in (None, [glob, loc, (loc + 2) % n, glob, 1], [glob]):
        got = grp.sample(400, base_seed=9, qubits=qubits)
        qs = list(range(n)) if qubits is None else qubits
        assert np.array_equal(got, oracle.tree_sample(probs, n, qs, 9, 400)), qubits
    assert grp.sample(0).size == 0
    with pytest.raises(Exception):
        grp.measure(n)
