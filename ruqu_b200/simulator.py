"""Stateless simulator entry points (crates/ruqu-core/src/simulator.rs:14-164)."""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from .circuit import QuantumCircuit
from .gate import GateKind
from .state import QuantumState
from .types import SimulationMetrics


@dataclass
class SimConfig:
    """simulator.rs:14-21, plus the amplitude precision of the GPU state."""

    seed: int | None = None
    noise: object = None
    shots: int | None = None
    precision: str = "f64"


@dataclass
class SimulationResult:
    state: QuantumState
    measurements: list
    metrics: SimulationMetrics


@dataclass
class ShotResult:
    counts: dict = field(default_factory=dict)   # tuple(bool per qubit) -> count
    metrics: SimulationMetrics = field(default_factory=SimulationMetrics)


def _metrics(n: int, gates: int, ns: int, precision: str) -> SimulationMetrics:
    secs = ns / 1e9
    return SimulationMetrics(num_qubits=n, gate_count=gates, execution_time_ns=ns,
                             peak_memory_bytes=QuantumState.estimate_memory(n, precision),
                             gates_per_second=gates / secs if secs > 0 else 0.0, gates_fused=0)


class Simulator:
    @staticmethod
    def run(circuit: QuantumCircuit) -> SimulationResult:
        return Simulator.run_with_config(circuit, SimConfig())

    @staticmethod
    def run_with_config(circuit: QuantumCircuit, config: SimConfig) -> SimulationResult:
        """simulator.rs:56-101: fresh |0...0>, every gate in order, metrics; with
        config.noise (a NoiseModel) the Pauli noise of apply_noise after every gate."""
        t0 = time.perf_counter_ns()
        state = QuantumState(circuit.num_qubits(), config.seed, config.precision)
        if not circuit.gate_count():
            meas = []
        elif config.noise is not None:
            meas = state.apply_gates_noisy(circuit.packed(), config.noise)
        else:
            meas = state.apply_gates(circuit.packed())
        state.synchronize()
        ns = time.perf_counter_ns() - t0
        unitary = sum(1 for g in circuit.gates() if not g.is_non_unitary())
        return SimulationResult(state, meas, _metrics(circuit.num_qubits(), unitary, ns, config.precision))

    @staticmethod
    def run_shots(circuit: QuantumCircuit, shots: int, seed: int | None = None,
                  precision: str = "f64") -> ShotResult:
        """simulator.rs:107-164.

        Shot s behaves as a fresh run with seed ``base + s`` (base 42 when
        ``seed`` is None), followed by ``measure_all`` when the circuit has no
        Measure gate.  When all Measure gates trail the unitary part and
        there is no Reset, the circuit is simulated once and every shot is
        drawn from the final state with exactly those seeds and draw order;
        otherwise each shot is re-simulated on the GPU.
        """
        t0 = time.perf_counter_ns()
        n = circuit.num_qubits()
        base = 42 if seed is None else int(seed)
        gates = circuit.gates()
        has_meas = any(g.kind == GateKind.Measure for g in gates)
        has_reset = any(g.kind == GateKind.Reset for g in gates)
        first_meas = next((k for k, g in enumerate(gates) if g.kind == GateKind.Measure), len(gates))
        trailing = all(g.kind in (GateKind.Measure, GateKind.Barrier) for g in gates[first_meas:])
        counts: dict = {}
        unitary = sum(1 for g in gates if not g.is_non_unitary())
        if not has_reset and trailing:
            body = gates[:first_meas]
            order = [g.q0 for g in gates[first_meas:] if g.kind == GateKind.Measure] if has_meas else list(range(n))
            state = QuantumState(n, 0, precision)
            if body:
                state.apply_gates(body)
            bits = state.sample(shots, base, order)
            measured = sorted(set(order))
            vals, cnt = np.unique(bits, return_counts=True)
            for v, c in zip(vals.tolist(), cnt.tolist()):
                key = tuple(bool((v >> q) & 1) if q in measured else False for q in range(n))
                counts[key] = counts.get(key, 0) + int(c)
        else:
            for s in range(int(shots)):
                state = QuantumState(n, (base + s) & (2**64 - 1), precision)
                meas = state.apply_gates(circuit.packed())
                if not has_meas:
                    meas += state.measure_all()
                b = [False] * n
                for m in meas:
                    if m.qubit < n:
                        b[m.qubit] = m.result
                counts[tuple(b)] = counts.get(tuple(b), 0) + 1
        ns = time.perf_counter_ns() - t0
        return ShotResult(counts, _metrics(n, unitary * int(shots), ns, precision))
