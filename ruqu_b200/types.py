"""Quantum-domain types (crates/ruqu-core/src/types.rs:182-263).

Amplitudes use Python/numpy complex numbers; the reference's own `Complex`
struct (types.rs:8-180) has no counterpart beyond that.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field


class PauliOp(enum.IntEnum):
    """types.rs:190-197; values match rq_pauli in include/ruqu_cuda.h."""

    I = 0
    X = 1
    Y = 2
    Z = 3


@dataclass
class PauliString:
    """Sparse tensor product of Pauli factors (types.rs:199-216)."""

    ops: list = field(default_factory=list)   # [(qubit, PauliOp)]

    @staticmethod
    def identity() -> "PauliString":
        return PauliString([])


@dataclass
class Hamiltonian:
    """Weighted sum of Pauli strings (types.rs:218-228)."""

    terms: list      # [(coeff, PauliString)]
    num_qubits: int


@dataclass
class MeasurementOutcome:
    """types.rs:230-235."""

    qubit: int
    result: bool
    probability: float


@dataclass
class SimulationMetrics:
    """types.rs:238-245."""

    num_qubits: int = 0
    gate_count: int = 0
    execution_time_ns: int = 0
    peak_memory_bytes: int = 0
    gates_per_second: float = 0.0
    gates_fused: int = 0


@dataclass
class NoiseModel:
    """types.rs:249-263: per-gate stochastic Pauli noise for Simulator.run_with_config."""

    depolarizing_rate: float = 0.0
    bit_flip_rate: float = 0.0
    phase_flip_rate: float = 0.0
