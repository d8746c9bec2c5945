"""VQE on the GPU state (crates/ruqu-algorithms/src/vqe.rs:25-282)."""
from __future__ import annotations

import math
from dataclasses import dataclass

from .circuit import QuantumCircuit
from .simulator import SimConfig, Simulator
from .types import Hamiltonian, PauliOp, PauliString


@dataclass
class VqeConfig:
    """vqe.rs:25-42 (plus the GPU state precision)."""

    hamiltonian: Hamiltonian
    num_qubits: int
    ansatz_depth: int
    max_iterations: int
    convergence_threshold: float
    learning_rate: float
    seed: int | None = None
    precision: str = "f64"


@dataclass
class VqeResult:
    optimal_energy: float
    optimal_parameters: list
    energy_history: list
    num_iterations: int
    converged: bool


def num_parameters(num_qubits: int, depth: int) -> int:
    """vqe.rs:65-67: Ry + Rz per qubit per layer."""
    return 2 * num_qubits * depth


def build_ansatz(num_qubits: int, depth: int, params) -> QuantumCircuit:
    """Per layer: Ry on all qubits, Rz on all qubits, CNOT chain (vqe.rs:81-112)."""
    expected = num_parameters(num_qubits, depth)
    if len(params) != expected:
        raise ValueError(f"build_ansatz: expected {expected} parameters, got {len(params)}")
    c = QuantumCircuit(num_qubits)
    k = 0
    for _ in range(depth):
        for q in range(num_qubits):
            c.ry(q, params[k])
            k += 1
        for q in range(num_qubits):
            c.rz(q, params[k])
            k += 1
        for q in range(max(0, num_qubits - 1)):
            c.cnot(q, q + 1)
    return c


def evaluate_energy(config: VqeConfig, params) -> float:
    """<psi(params)|H|psi(params)> (vqe.rs:122-131)."""
    circuit = build_ansatz(config.num_qubits, config.ansatz_depth, params)
    res = Simulator.run_with_config(circuit, SimConfig(seed=config.seed, precision=config.precision))
    return res.state.expectation_hamiltonian(config.hamiltonian)


def run_vqe(config: VqeConfig) -> VqeResult:
    """Parameter-shift gradient descent from params = 0.1 (vqe.rs:148-216)."""
    n_params = num_parameters(config.num_qubits, config.ansatz_depth)
    params = [0.1] * n_params
    hist = []
    converged = False
    best = 1.7976931348623157e308
    best_params = list(params)
    shift = math.pi / 2
    for it in range(config.max_iterations):
        e = evaluate_energy(config, params)
        hist.append(e)
        if e < best:
            best = e
            best_params = list(params)
        if it > 0 and abs(hist[it - 1] - e) < config.convergence_threshold:
            converged = True
            break
        grad = [0.0] * n_params
        for i in range(n_params):
            pp, pm = list(params), list(params)
            pp[i] += shift
            pm[i] -= shift
            grad[i] = (evaluate_energy(config, pp) - evaluate_energy(config, pm)) / 2.0
        for i in range(n_params):
            params[i] -= config.learning_rate * grad[i]
    return VqeResult(best, best_params, hist, len(hist), converged)


def h2_hamiltonian() -> Hamiltonian:
    """2-qubit H2 Hamiltonian of vqe.rs:257-272 (ground energy about -1.137 Ha)."""
    return Hamiltonian([
        (-1.0523, PauliString([])),
        (0.3979, PauliString([(1, PauliOp.Z)])),
        (-0.3979, PauliString([(0, PauliOp.Z)])),
        (-0.0112, PauliString([(0, PauliOp.Z), (1, PauliOp.Z)])),
        (0.1809, PauliString([(0, PauliOp.X), (1, PauliOp.X)])),
    ], 2)


def single_z_hamiltonian() -> Hamiltonian:
    """H = -Z on one qubit (vqe.rs:277-282)."""
    return Hamiltonian([(-1.0, PauliString([(0, PauliOp.Z)]))], 1)
