"""QAOA for MaxCut on the GPU state (crates/ruqu-algorithms/src/qaoa.rs:34-308)."""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .circuit import QuantumCircuit
from .simulator import SimConfig, Simulator
from .types import PauliOp, PauliString


@dataclass
class Graph:
    """qaoa.rs:34-75."""

    num_nodes: int
    edges: list = field(default_factory=list)   # [(i, j, w)]

    def add_edge(self, i: int, j: int, weight: float) -> None:
        if i >= self.num_nodes:
            raise IndexError(f"node index {i} out of range")
        if j >= self.num_nodes:
            raise IndexError(f"node index {j} out of range")
        self.edges.append((i, j, float(weight)))

    @staticmethod
    def unweighted(num_nodes: int, edges) -> "Graph":
        return Graph(num_nodes, [(int(i), int(j), 1.0) for i, j in edges])

    def num_edges(self) -> int:
        return len(self.edges)


@dataclass
class QaoaConfig:
    """qaoa.rs:82-93 (plus the GPU state precision)."""

    graph: Graph
    p: int
    max_iterations: int
    learning_rate: float
    seed: int | None = None
    precision: str = "f64"


@dataclass
class QaoaResult:
    best_cut_value: float
    best_bitstring: list
    optimal_gammas: list
    optimal_betas: list
    energy_history: list
    converged: bool


def build_qaoa_circuit(graph: Graph, gammas, betas) -> QuantumCircuit:
    """H on every qubit, then per layer Rzz(2*gamma*w) per edge and Rx(2*beta) per qubit (qaoa.rs:125-153)."""
    if len(gammas) != len(betas):
        raise ValueError("gammas and betas must have equal length")
    c = QuantumCircuit(graph.num_nodes)
    for q in range(graph.num_nodes):
        c.h(q)
    for layer in range(len(gammas)):
        for i, j, w in graph.edges:
            c.rzz(i, j, 2.0 * gammas[layer] * w)
        for q in range(graph.num_nodes):
            c.rx(q, 2.0 * betas[layer])
    return c


def cut_value(graph: Graph, bitstring) -> float:
    """qaoa.rs:162-169."""
    return sum(w for i, j, w in graph.edges if bool(bitstring[i]) != bool(bitstring[j]))


def evaluate_qaoa_cost(graph: Graph, gammas, betas, seed=None, precision="f64") -> float:
    """sum_edges w * (1 - <Z_i Z_j>) / 2 (qaoa.rs:179-201); all <ZZ> in one device pass."""
    circuit = build_qaoa_circuit(graph, gammas, betas)
    res = Simulator.run_with_config(circuit, SimConfig(seed=seed, precision=precision))
    zz = res.state.expectation_values([PauliString([(i, PauliOp.Z), (j, PauliOp.Z)]) for i, j, _ in graph.edges])
    cost = 0.0
    for (i, j, w), z in zip(graph.edges, zz):
        cost += w * 0.5 * (1.0 - z)
    return cost


WASM_MAX_QUBITS = 25


def qaoa_maxcut(num_nodes: int, edges_flat, p: int, gammas, betas, seed=None, precision: str = "f64") -> dict:
    """ruqu-wasm's qaoa_maxcut by semantics (crates/ruqu-wasm/src/lib.rs:408-500): a graph
    from flattened (u, v) pairs with unit weights, the QAOA circuit of build_qaoa_circuit,
    one run_with_config, then {"probabilities": all 2^n probabilities, "expected_cut":
    sum over the listed pairs of (1 - <Z_u Z_v>) / 2}.  The same argument checks (at most
    25 nodes, p angles each, an even number of node indices), raised as ValueError; the
    <ZZ> of all pairs come from one device call."""
    if num_nodes > WASM_MAX_QUBITS:
        raise ValueError(f"Qubit limit exceeded: {num_nodes} requested, max {WASM_MAX_QUBITS} in WASM")
    gammas = list(gammas)
    betas = list(betas)
    if len(gammas) != p:
        raise ValueError(f"gammas length mismatch: expected {p} (p), got {len(gammas)}")
    if len(betas) != p:
        raise ValueError(f"betas length mismatch: expected {p} (p), got {len(betas)}")
    edges_flat = [int(x) for x in edges_flat]
    if len(edges_flat) % 2:
        raise ValueError("edges_flat must contain an even number of elements (pairs of node indices)")
    graph = Graph(num_nodes)
    pairs = list(zip(edges_flat[0::2], edges_flat[1::2]))
    for u, v in pairs:
        graph.add_edge(u, v, 1.0)
    res = Simulator.run_with_config(build_qaoa_circuit(graph, gammas, betas), SimConfig(seed=seed, precision=precision))
    probs = res.state.probabilities()
    zz = res.state.expectation_values([PauliString([(u, PauliOp.Z), (v, PauliOp.Z)]) for u, v in pairs]) if pairs else []
    expected_cut = 0.0
    for z in zz:
        expected_cut += 0.5 * (1.0 - z)
    return {"probabilities": probs, "expected_cut": float(expected_cut)}


def _best_index(probs: np.ndarray) -> int:
    """Iterator::max_by semantics: the last of equal maxima (qaoa.rs:249-255)."""
    mx = probs.max()
    return int(np.flatnonzero(probs == mx)[-1])


def run_qaoa(config: QaoaConfig) -> QaoaResult:
    """Gradient ascent with the parameter-shift rule from gamma = beta = 0.5 (qaoa.rs:217-308)."""
    p = config.p
    g = [0.5] * p
    b = [0.5] * p
    hist = []
    best = -math.inf
    best_bits = [False] * config.graph.num_nodes
    converged = False
    shift = math.pi / 2
    for it in range(config.max_iterations):
        cost = evaluate_qaoa_cost(config.graph, g, b, config.seed, config.precision)
        hist.append(cost)
        if cost > best:
            best = cost
            res = Simulator.run_with_config(build_qaoa_circuit(config.graph, g, b),
                                            SimConfig(seed=config.seed, precision=config.precision))
            idx = _best_index(res.state.probabilities())
            best_bits = [bool((idx >> q) & 1) for q in range(config.graph.num_nodes)]
        if it > 0 and abs(cost - hist[it - 1]) < 1e-6:
            converged = True
            break
        for i in range(p):
            gp, gm = list(g), list(g)
            gp[i] += shift
            gm[i] -= shift
            cp = evaluate_qaoa_cost(config.graph, gp, b, config.seed, config.precision)
            cm = evaluate_qaoa_cost(config.graph, gm, b, config.seed, config.precision)
            g[i] += config.learning_rate * (cp - cm) / 2.0
        for i in range(p):
            bp, bm = list(b), list(b)
            bp[i] += shift
            bm[i] -= shift
            cp = evaluate_qaoa_cost(config.graph, g, bp, config.seed, config.precision)
            cm = evaluate_qaoa_cost(config.graph, g, bm, config.seed, config.precision)
            b[i] += config.learning_rate * (cp - cm) / 2.0
    return QaoaResult(best, best_bits, g, b, hist, converged)


def triangle_graph() -> Graph:
    return Graph.unweighted(3, [(0, 1), (1, 2), (0, 2)])


def ring4_graph() -> Graph:
    return Graph.unweighted(4, [(0, 1), (1, 2), (2, 3), (3, 0)])
