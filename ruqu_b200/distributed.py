"""A state vector split over ranks by its top qubits (a distributed state).

With 2^g ranks, each rank holds the 2^(n-g) amplitudes whose top g bits are its rank
index.  A layout maps every logical qubit to a physical bit: bits below n - g are
local (inside each rank's state), the top g are the rank's bits.  A gate whose
qubits are all local runs on every rank's state unchanged.  A diagonal gate on a
global qubit becomes, per rank, a local gate or a phase (the rank knows its own bit):
Rz / Phase / Z / S / T on a global qubit multiply the rank's state by one of the two
diagonal entries; CZ / Rzz / CNOT controls on global qubits turn into a local Z / Rz
/ X or a phase.  Any other gate on a global qubit first makes it local: it swaps
places with a local qubit, each rank sending the half of its amplitudes whose local
bit differs from its own global bit to the partner rank (rank ^ 2^j) and receiving
the partner's half in its place (`rq_state_half_copy` packs and unpacks on the
device).  The local qubit given up is the one whose next use lies furthest ahead.
A SWAP gate only relabels the layout.

Measurement, reset and shots follow state.rs:288-352 and simulator.rs:107-147 on the
whole state: each rank reduces its own amplitudes, the ranks add their shares, and every
rank takes the same draw of one measurement stream (Philox key = the state's seed), so
all ranks reach the same outcome and collapse their own amplitudes.  Shots walk the
sampler's prefix tree: each rank keeps the tree of its local qubits, and every step of
the walk adds the ranks' shares of the conditional probabilities of all shots at once.

The schedule (local runs and swaps) depends on the gate list and the layout alone,
so every rank computes the same one; the per-rank translation of a local run depends
on the rank's bits.  Executors: `DistributedState` runs one rank per process (SPMD,
`torch.distributed` send / receive of the packed halves: NCCL between GPUs), and
`StateGroup` runs all ranks in one process (every rank's state in this process;
the halves swap by buffer).  The reference has no distributed state (its largest
dense state is one host vector); this is the multi-GPU step that follows the
single-GPU path once a state outgrows one GPU.
"""
from __future__ import annotations

import cmath
import math

import numpy as np

from .error import InvalidQubitIndex
from .gate import Gate
from .rng import uniforms, uniforms_keys
from .types import MeasurementOutcome

H, X, Y, Z, S, SDG, T, TDG, RX, RY, RZ, PHASE, CNOT, CZ, SWAP, RZZ, MEASURE, RESET, BARRIER, U1 = range(20)
_DIAG_1Q = (Z, S, SDG, T, TDG, RZ, PHASE)
_NONDIAG_1Q = (H, X, Y, RX, RY, U1)


def _as_tuple(g):
    t = g.to_tuple() if isinstance(g, Gate) else tuple(g)
    kind, q0 = int(t[0]), int(t[1])
    q1 = int(t[2]) if len(t) > 2 else 0
    angle = float(t[3]) if len(t) > 3 else 0.0
    m = t[4] if len(t) > 4 else None
    return (kind, q0, q1, angle, m)


def diagonal_entries(kind: int, angle: float):
    """(d0, d1) of a diagonal 1-qubit gate (the matrices of gate.rs:72-146)."""
    if kind == Z:
        return 1.0, -1.0
    if kind == S:
        return 1.0, 1j
    if kind == SDG:
        return 1.0, -1j
    if kind == T:
        return 1.0, cmath.exp(1j * math.pi / 4)
    if kind == TDG:
        return 1.0, cmath.exp(-1j * math.pi / 4)
    if kind == RZ:
        return cmath.exp(-0.5j * angle), cmath.exp(0.5j * angle)
    if kind == PHASE:
        return 1.0, cmath.exp(1j * angle)
    raise ValueError(f"gate kind {kind} is not diagonal")


def _needs_local(g):
    """Logical qubits that must be local for the gate (the rest may stay global)."""
    kind, q0, q1 = g[0], g[1], g[2]
    if kind in _NONDIAG_1Q:
        return (q0,)
    if kind == CNOT:
        return (q1,)
    return ()


class Layout:
    """Logical qubit -> physical bit for n qubits over 2^g ranks."""

    def __init__(self, num_qubits: int, global_qubits: int):
        if not 0 <= global_qubits < num_qubits:
            raise ValueError("need 0 <= global qubits < qubits")
        self.n, self.g = int(num_qubits), int(global_qubits)
        self.nl = self.n - self.g
        self.phys = list(range(self.n))      # logical -> physical
        self.logical = list(range(self.n))   # physical -> logical

    def is_local(self, q: int) -> bool:
        return self.phys[q] < self.nl

    def exchange(self, pa: int, pb: int) -> None:
        """The logical qubits at physical bits pa and pb trade places."""
        la, lb = self.logical[pa], self.logical[pb]
        self.logical[pa], self.logical[pb] = lb, la
        self.phys[la], self.phys[lb] = pb, pa

    def copy(self) -> "Layout":
        c = Layout(self.n, self.g)
        c.phys, c.logical = list(self.phys), list(self.logical)
        return c


def schedule(gates, layout: Layout):
    """Steps for the gate list from the given layout (updated in place):
    ("local", [gates with physical qubits]) and ("swap", local bit, global bit j)."""
    gl = [_as_tuple(g) for g in gates]
    for g in gl:
        if g[0] in (MEASURE, RESET):
            raise ValueError("a schedule holds unitary gates only (apply_gates runs Measure / Reset)")
        if g[0] > U1:
            raise ValueError(f"unsupported gate kind {g[0]}")
    steps = []
    run = []

    def flush():
        if run:
            steps.append(("local", list(run)))
            run.clear()

    # the position of each gate's required-local qubits, for choosing which local qubit to give up
    uses = {}
    for k, g in enumerate(gl):
        for q in _needs_local(g):
            uses.setdefault(q, []).append(k)
    ptr = {q: 0 for q in uses}

    def next_use(q, k):
        lst = uses.get(q, [])
        i = ptr.get(q, 0)
        while i < len(lst) and lst[i] < k:
            i += 1
        ptr[q] = i
        return lst[i] if i < len(lst) else math.inf

    for k, g in enumerate(gl):
        kind = g[0]
        if kind == BARRIER:
            continue
        if kind == SWAP:
            layout.exchange(layout.phys[g[1]], layout.phys[g[2]])
            continue
        for q in _needs_local(g):
            if layout.is_local(q):
                continue
            busy = {layout.phys[x] for x in (g[1], g[2]) if layout.is_local(x)}
            victim, far = None, -1.0
            for p in range(layout.nl - 1, -1, -1):
                if p in busy:
                    continue
                nu = next_use(layout.logical[p], k)
                if nu > far:
                    victim, far = p, nu
            j = layout.phys[q] - layout.nl
            flush()
            steps.append(("swap", victim, j))
            layout.exchange(victim, layout.phys[q])
        run.append((kind, layout.phys[g[1]], layout.phys[g[2]], g[3], g[4]))
    flush()
    return steps


def translate(run, nl: int, rank: int):
    """One rank's local gates for a run of physically placed gates, plus the scalar
    phase the run multiplies this rank's state by (from diagonal factors on global bits)."""
    out = []
    phase = 1.0 + 0.0j

    def bit(p):
        return (rank >> (p - nl)) & 1

    for kind, p0, p1, angle, m in run:
        g0 = p0 >= nl
        two = kind in (CNOT, CZ, RZZ)
        g1 = two and p1 >= nl
        if not g0 and not g1:
            out.append((kind, p0, p1, angle, m) if m is not None else (kind, p0, p1, angle))
            continue
        if kind in _DIAG_1Q:
            d0, d1 = diagonal_entries(kind, angle)
            phase *= d1 if bit(p0) else d0
        elif kind == CZ:
            if g0 and g1:
                if bit(p0) and bit(p1):
                    phase *= -1.0
            elif g0:
                if bit(p0):
                    out.append((Z, p1, 0, 0.0))
            elif bit(p1):
                out.append((Z, p0, 0, 0.0))
        elif kind == RZZ:
            if g0 and g1:
                phase *= cmath.exp(-0.5j * angle) if bit(p0) == bit(p1) else cmath.exp(0.5j * angle)
            else:
                v, loc = (bit(p0), p1) if g0 else (bit(p1), p0)
                out.append((RZ, loc, 0, angle if v == 0 else -angle))
        elif kind == CNOT and g0 and not g1:
            if bit(p0):
                out.append((X, p1, 0, 0.0))
        else:
            raise AssertionError("a gate needing a local qubit reached a run with it global")
    return out, phase


def _phase_gate(phase: complex):
    """A Unitary1Q on local qubit 0 multiplying every amplitude by `phase`."""
    return (U1, 0, 0, 0.0, [phase.real, phase.imag, 0.0, 0.0, 0.0, 0.0, phase.real, phase.imag])


class DeviceRank:
    """One rank's local state on the current GPU (QuantumState of the local qubits) with
    two device buffers of half a state for the exchanges."""

    def __init__(self, local_qubits: int, seed: int = 0, precision: str = "f64"):
        import torch

        from .state import QuantumState
        self._torch = torch
        self.state = QuantumState(local_qubits, seed, precision)
        half = (1 << (local_qubits - 1)) * (8 if precision == "f32" else 16)
        self._send = torch.empty(half, dtype=torch.uint8, device="cuda")
        self._recv = torch.empty(half, dtype=torch.uint8, device="cuda")

    def apply(self, gates) -> None:
        if gates:
            self.state.apply_gates(gates)

    def zero(self) -> None:
        self.state.apply_gates([(U1, 0, 0, 0.0, [0.0] * 8)])

    def pack(self, p: int, v: int):
        self.state.half_copy(p, v, self._send.data_ptr())
        self.state.synchronize()          # the buffer is read on torch's streams next
        return self._send

    def recv_buffer(self):
        return self._recv

    def unpack(self, p: int, v: int, buf) -> None:
        self._torch.cuda.synchronize()    # the buffer was written on torch's streams
        self.state.half_copy(p, v, buf.data_ptr(), unpack=True)

    def expectation(self, strings) -> np.ndarray:
        return self.state.expectation_values(strings)

    def tree_build(self, bits) -> None:
        self.state.tree_build(bits)

    def tree_lookup(self, level: int, index) -> np.ndarray:
        return self.state.tree_lookup(level, index)

    def amplitudes(self) -> np.ndarray:
        return self.state.state_vector()


class _Distributed:
    """Layout bookkeeping and gate / expectation logic shared by the executors."""

    def _init_layout(self, num_qubits: int, global_qubits: int, seed: int = 0):
        self.layout = Layout(num_qubits, global_qubits)
        self.n, self.nl = self.layout.n, self.layout.nl
        self.seed = int(seed) & (2**64 - 1)   # the measurement stream (stream 0 of this key)
        self.draws = 0
        self.measurement_record = []

    def _localize(self, qubits) -> None:
        """Make the given logical qubits local (swapping out local qubits not among them)."""
        keep = set(qubits)
        for q in qubits:
            if self.layout.is_local(q):
                continue
            victim = next(p for p in range(self.nl - 1, -1, -1) if self.layout.logical[p] not in keep)
            j = self.layout.phys[q] - self.nl
            self._swap(victim, j)
            self.layout.exchange(victim, self.layout.phys[q])

    def apply_gates(self, gates) -> list:
        """The gates in order (QuantumState::apply_gate, state.rs:158-204): unitary runs
        through the schedule, Measure / Reset through measure / reset_qubit; returns the
        measurement outcomes."""
        outcomes, run = [], []
        for g in gates:
            t = _as_tuple(g)
            if t[0] in (MEASURE, RESET):
                self._apply_unitary(run)
                run = []
                if t[0] == MEASURE:
                    outcomes.append(self.measure(t[1]))
                else:
                    self.reset_qubit(t[1])
            else:
                run.append(g)
        self._apply_unitary(run)
        return outcomes

    def _apply_unitary(self, gates) -> None:
        if not gates:
            return
        for step in schedule(gates, self.layout):
            if step[0] == "swap":
                self._swap(step[1], step[2])
            else:
                self._run_local(step[1])

    def _local_strings(self, strings, rank: int):
        """Each string's factors on local qubits (physical indices) and the sign its Z
        factors on global qubits give this rank."""
        out, signs = [], []
        for st in strings:
            loc, sign = [], 1.0
            for q, op in st:
                op = int(op)
                if op == 0:
                    continue
                p = self.layout.phys[int(q)]
                if p < self.nl:
                    loc.append((p, op))
                elif (rank >> (p - self.nl)) & 1:   # Z on a global qubit (X / Y were made local)
                    sign = -sign
            out.append(loc)
            signs.append(sign)
        return out, np.asarray(signs)

    def _string_groups(self, strings):
        """The strings in groups whose flipped (X / Y) qubits fit in one rank's local
        qubits together; yields (positions, strings) after making each group's flipped
        qubits local."""
        strings = [[(int(q), int(op)) for q, op in st] for st in strings]
        groups, cur, cur_flips = [], [], set()
        for k, st in enumerate(strings):
            for q, _ in st:
                if not 0 <= q < self.n:
                    raise ValueError(f"qubit {q} out of range for {self.n} qubits")
            f = {q for q, op in st if op in (1, 2)}
            if len(f) > self.nl:
                raise ValueError("a string flips more qubits than one rank holds")
            if cur and len(cur_flips | f) > self.nl:
                groups.append((cur, cur_flips))
                cur, cur_flips = [], set()
            cur.append(k)
            cur_flips |= f
        if cur:
            groups.append((cur, cur_flips))
        for idx, flips in groups:
            self._localize(sorted(flips))
            yield idx, [strings[k] for k in idx]

    # ---- measurement (state.rs:288-352) and shots (simulator.rs:107-147) ----
    def _check_qubit(self, q: int) -> int:
        q = int(q)
        if not 0 <= q < self.n:
            raise InvalidQubitIndex(f"invalid qubit index {q} for {self.n}-qubit system")
        return q

    def measure(self, qubit: int) -> MeasurementOutcome:
        """QuantumState::measure (state.rs:288-326) on the whole distributed state:
        p0 = sum over every rank of |a|^2 with the qubit 0 (FP64), the next draw u of
        the measurement stream, outcome = u >= p0, probability = 1 - p0 or p0, and
        the collapse scaled by 1/sqrt(probability) (0 for a zero probability).  A local
        qubit is one reduction per rank and a projector on it; a global qubit is each
        rank's norm, and the ranks on the other side of the outcome are zeroed."""
        q = self._check_qubit(qubit)
        p = self.layout.phys[q]
        if p < self.nl:
            def part(r, eng):
                i, z = eng.expectation([[], [(p, 3)]])
                return np.array([0.5 * (float(i) + float(z))])
        else:
            j = p - self.nl

            def part(r, eng):
                return np.array([0.0 if (r >> j) & 1 else float(eng.expectation([[]])[0])])
        p0 = float(self._rank_sum(part)[0])
        u = float(uniforms(self.seed, 0, self.draws, 1)[0])
        self.draws += 1
        result = u >= p0
        prob = 1.0 - p0 if result else p0
        f = 1.0 / math.sqrt(prob) if prob > 0.0 else 0.0
        for r, eng in self._local_ranks():
            if p < self.nl:
                m = [0.0, 0.0, 0.0, 0.0, 0.0, 0.0, f, 0.0] if result else [f, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0]
                eng.apply([(U1, p, 0, 0.0, m)])
            elif ((r >> j) & 1) == int(result):
                eng.apply([_phase_gate(complex(f))])
            else:
                eng.zero()
        out = MeasurementOutcome(q, bool(result), prob)
        self.measurement_record.append(out)
        return out

    def measure_all(self) -> list:
        """Qubit 0 first (state.rs:329-335)."""
        return [self.measure(q) for q in range(self.n)]

    def reset_qubit(self, qubit: int) -> None:
        """Measure, then X if the outcome was 1 (state.rs:340-350)."""
        if self.measure(qubit).result:
            self.apply_gates([(X, int(qubit), 0, 0.0)])

    def sample(self, shots: int, base_seed: int = 42, qubits=None) -> np.ndarray:
        """Shot bitstrings without collapse, as QuantumState.sample / rq_state_sample: shot s
        measures ``qubits`` in order with draws 0, 1, ... of key base_seed + s, outcome 1
        iff u >= P(qubit = 0 | earlier outcomes) (simulator.rs:107-147, state.rs:288-304).
        Each rank builds the prefix tree of its local qubits in measurement order; at step
        k every rank looks up its share of P(prefix, 0) and P(prefix, 1) for every shot (a
        global qubit: its rank bit splits the ranks' shares; ranks whose bits contradict a
        shot's global outcomes add nothing) and the shares are summed over ranks (one
        all-reduce of 2 x shots doubles per measured qubit).  Every rank walks the same
        shots to the same bitstrings.  Sums over ranks round differently from one tree over
        the whole state, so a shot can differ from the one-GPU sampler only where its draw
        falls within rounding of its conditional probability."""
        qs = list(range(self.n)) if qubits is None else [self._check_qubit(q) for q in qubits]
        if len(qs) > 64:
            raise ValueError("at most 64 measurements per shot")
        shots = int(shots)
        out = np.zeros(shots, dtype=np.uint64)
        if shots == 0 or not qs:
            return out
        pos = {}
        for q in qs:
            p = self.layout.phys[q]
            if p < self.nl and p not in pos:
                pos[p] = len(pos)
        order = sorted(pos, key=pos.get)
        for _, eng in self._local_ranks():
            eng.tree_build(order)
        keys = np.uint64(int(base_seed) & (2**64 - 1)) + np.arange(shots, dtype=np.uint64)
        prefix = np.zeros(shots, dtype=np.uint64)
        ok = {r: np.ones(shots, dtype=bool) for r, _ in self._local_ranks()}
        zeros = np.zeros(shots)
        lvl = 0
        val = {}
        for k, q in enumerate(qs):
            if q not in val:
                p = self.layout.phys[q]
                if p < self.nl:
                    b = np.uint64(1) << np.uint64(pos[p])

                    def part(r, eng):
                        v0 = eng.tree_lookup(lvl + 1, prefix)
                        v1 = eng.tree_lookup(lvl + 1, prefix | b)
                        return np.concatenate([np.where(ok[r], v0, 0.0), np.where(ok[r], v1, 0.0)])
                else:
                    j = p - self.nl

                    def part(r, eng):
                        v = np.where(ok[r], eng.tree_lookup(lvl, prefix), 0.0)
                        return np.concatenate([zeros, v] if (r >> j) & 1 else [v, zeros])
                m = self._rank_sum(part)
                m0, m1 = m[:shots], m[shots:]
                with np.errstate(invalid="ignore", divide="ignore"):
                    p0 = m0 / (m0 + m1)
                res = uniforms_keys(keys, 0, k) >= p0
                if p < self.nl:
                    prefix |= res.astype(np.uint64) << np.uint64(pos[p])
                    lvl += 1
                else:
                    for r in ok:
                        ok[r] &= res == bool((r >> j) & 1)
                val[q] = res
            bit = np.uint64(1) << np.uint64(q)
            out = np.where(val[q], out | bit, out & ~bit)
        return out

    def _logical_order(self, phys_amps: np.ndarray) -> np.ndarray:
        """Amplitudes in physical index order -> logical index order."""
        n = self.n
        idx = np.arange(1 << n, dtype=np.int64)
        src = np.zeros_like(idx)
        for q in range(n):
            src |= ((idx >> q) & 1) << self.layout.phys[q]
        return phys_amps[src]


class StateGroup(_Distributed):
    """All 2^g ranks of a distributed state in this process (one engine per rank, e.g.
    several DeviceRank states on one GPU); exchanges swap the packed halves directly."""

    def __init__(self, num_qubits: int, global_qubits: int, precision: str = "f64", seed: int = 0,
                 engines=None):
        self._init_layout(num_qubits, global_qubits, seed)
        w = 1 << global_qubits
        self.ranks = list(engines) if engines is not None else [DeviceRank(self.nl, seed, precision)
                                                                 for _ in range(w)]
        if len(self.ranks) != w:
            raise ValueError(f"{w} ranks needed")
        for r in range(1, w):
            self.ranks[r].zero()

    def _local_ranks(self):
        return list(enumerate(self.ranks))

    def _rank_sum(self, fn) -> np.ndarray:
        """The sum over ranks (in rank order) of fn(rank, engine)."""
        total = None
        for r, eng in enumerate(self.ranks):
            v = np.asarray(fn(r, eng), dtype=np.float64)
            total = v.copy() if total is None else total + v
        return total

    def _run_local(self, run) -> None:
        for r, eng in enumerate(self.ranks):
            gl, ph = translate(run, self.nl, r)
            if ph != 1.0:
                gl.append(_phase_gate(ph))
            eng.apply(gl)

    def _swap(self, p: int, j: int) -> None:
        for r in range(len(self.ranks)):
            if (r >> j) & 1:
                continue
            q = r | (1 << j)
            a = self.ranks[r].pack(p, 1)   # rank r (bit j = 0) sends its bit-p = 1 half
            b = self.ranks[q].pack(p, 0)   # the partner (bit j = 1) sends its bit-p = 0 half
            self.ranks[r].unpack(p, 1, b)
            self.ranks[q].unpack(p, 0, a)

    def expectation_values(self, strings) -> np.ndarray:
        total = np.zeros(len(strings))
        for idx, group in self._string_groups(strings):
            for r, eng in enumerate(self.ranks):
                loc, signs = self._local_strings(group, r)
                total[idx] += signs * np.asarray(eng.expectation(loc), dtype=np.float64)
        return total

    def state_vector(self) -> np.ndarray:
        return self._logical_order(np.concatenate([eng.amplitudes() for eng in self.ranks]))


class DistributedState(_Distributed):
    """One rank of a distributed state per process (torchrun, one GPU each): 2^g ranks,
    the top g qubits global.  Exchanges are torch.distributed send / receive of the
    packed halves (NCCL between GPUs; gloo with host buffers); every rank must make the
    same calls in the same order."""

    def __init__(self, num_qubits: int, precision: str = "f64", seed: int = 0, engine=None):
        import torch.distributed as tdist
        self._dist = tdist
        self.rank, world = tdist.get_rank(), tdist.get_world_size()
        g = world.bit_length() - 1
        if 1 << g != world:
            raise ValueError("the number of ranks must be a power of two")
        self._init_layout(num_qubits, g, seed)
        self.engine = engine if engine is not None else DeviceRank(self.nl, seed, precision)
        if self.rank != 0:
            self.engine.zero()

    def _local_ranks(self):
        return [(self.rank, self.engine)]

    def _rank_sum(self, fn) -> np.ndarray:
        """fn(rank, engine) summed over the process group (all-reduce; the same on every rank)."""
        import torch

        from .dist import _device
        t = torch.tensor(np.asarray(fn(self.rank, self.engine), dtype=np.float64), dtype=torch.float64,
                         device=_device())
        self._dist.all_reduce(t)
        return t.cpu().numpy()

    def _run_local(self, run) -> None:
        gl, ph = translate(run, self.nl, self.rank)
        if ph != 1.0:
            gl.append(_phase_gate(ph))
        self.engine.apply(gl)

    def _swap(self, p: int, j: int) -> None:
        partner = self.rank ^ (1 << j)
        v = 1 - ((self.rank >> j) & 1)
        send = self.engine.pack(p, v)
        recv = self.engine.recv_buffer()
        reqs = [self._dist.isend(send, partner), self._dist.irecv(recv, partner)]
        for q in reqs:
            q.wait()
        self.engine.unpack(p, v, recv)

    def expectation_values(self, strings) -> np.ndarray:
        import torch

        from .dist import _device
        part = np.zeros(len(strings))
        for idx, group in self._string_groups(strings):
            loc, signs = self._local_strings(group, self.rank)
            part[idx] = signs * np.asarray(self.engine.expectation(loc), dtype=np.float64)
        t = torch.tensor(part, dtype=torch.float64, device=_device())
        self._dist.all_reduce(t)
        return t.cpu().numpy()

    def state_vector(self) -> np.ndarray:
        """The whole state in logical order on every rank (for small states)."""
        parts = [None] * self._dist.get_world_size()
        self._dist.all_gather_object(parts, self.engine.amplitudes())
        return self._logical_order(np.concatenate(parts))
