"""Grover search on the GPU state (crates/ruqu-algorithms/src/grover.rs).

The reference edits amplitudes on the host through amplitudes_mut for the oracle
and the middle of the diffuser; here those edits are device passes
(QuantumState.negate_amplitudes / negate_all_except), so the state never leaves
the GPU.  The Hadamard layers go through the gate pipeline as in the reference.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

from .gate import Gate
from .state import QuantumState


@dataclass
class GroverConfig:
    """grover.rs:27-39."""

    num_qubits: int
    target_states: list = field(default_factory=list)
    num_iterations: int | None = None
    seed: int | None = None
    precision: str = "f64"


@dataclass
class GroverResult:
    """grover.rs:42-53."""

    measured_state: int
    target_found: bool
    success_probability: float
    num_iterations: int
    state: QuantumState


def optimal_iterations(num_qubits: int, num_targets: int) -> int:
    """grover.rs:69-74: round(pi/4 / asin(sqrt(M/N)) - 1/2), at least 1.  With no
    targets the reference's count is infinite (saturating to u32::MAX); this raises."""
    if num_targets <= 0:
        raise ValueError("optimal_iterations needs at least one target state")
    n = 1 << num_qubits
    theta = math.asin(math.sqrt(num_targets / n))
    k = max(1.0, _round_half_away(math.pi / 4 / theta - 0.5))
    return int(k)


def _round_half_away(x: float) -> float:
    # f64::round rounds halves away from zero (Python's round() rounds them to even)
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


def run_grover(config: GroverConfig) -> GroverResult:
    """grover.rs:99-184: |s> = H^n|0>, then per iteration the oracle (negate the
    targets) and the diffuser (H^n, negate all but |0...0>, H^n); the success
    probability before measurement; every qubit measured in ascending order."""
    n = int(config.num_qubits)
    dim = 1 << n
    for t in config.target_states:
        if not 0 <= t < dim:
            raise ValueError(f"target state index {t} out of range for {n} qubits (max {dim - 1})")
    iterations = (config.num_iterations if config.num_iterations is not None
                  else optimal_iterations(n, len(config.target_states)))
    state = QuantumState(n, config.seed, config.precision)
    hs = [Gate.H(q) for q in range(n)]
    state.apply_gates(hs)
    for _ in range(iterations):
        state.negate_amplitudes(config.target_states)
        state.apply_gates(hs)
        state.negate_all_except(0)
        state.apply_gates(hs)
    probs = state.probabilities()
    success = float(sum(probs[t] for t in config.target_states))
    measured = 0
    for q in range(n):
        if state.measure(q).result:
            measured |= 1 << q
    return GroverResult(measured, measured in config.target_states, success, int(iterations), state)
