"""Seeded synthetic workloads of the state-vector path.

Every generator draws from the Philox stream of ``ruqu_b200.rng`` with a
documented stream id and draw order, so the same workload can be rebuilt
anywhere (host tests, the bench, the CPU baseline):

* stream 1 -- random-layer circuit angles: layer -> qubit -> (theta, phi)
* stream 2 -- random 3-regular graphs (pairing model with rejection)
* stream 3 -- QAOA instance sizes and angles
* stream 4 -- random Pauli-string Hamiltonians
* stream 5 -- VQE parameter sets

The reference ships no workload generators; these are compositions of its
circuit API (circuit.rs) and gate set (gate.rs).
"""
from __future__ import annotations

import math

import numpy as np

from .gate import GateKind
from .rng import Stream

TWO_PI = 2.0 * math.pi


def random_layer_circuit(n: int, layers: int, seed: int) -> list:
    """Per layer: Rz(theta_q) then Rx(phi_q) on every qubit q, theta, phi ~ U[0, 2pi);
    then CNOT(i, i+1) for even i on even layers and odd i on odd layers.
    Returns (kind, q0, q1, angle) tuples."""
    st = Stream(seed, 1)
    u = st.take(2 * n * layers).reshape(layers, n, 2) * TWO_PI
    gates = []
    for l in range(layers):
        for q in range(n):
            gates.append((int(GateKind.Rz), q, 0, float(u[l, q, 0])))
            gates.append((int(GateKind.Rx), q, 0, float(u[l, q, 1])))
        for i in range(l % 2, n - 1, 2):
            gates.append((int(GateKind.CNOT), i, i + 1, 0.0))
    return gates


def random_layer_bytes(n: int, layers: int, elem_bytes: int) -> int:
    """Algorithmic HBM bytes of the unfused circuit: 2S per 1-qubit gate, S per CNOT
    (a CNOT reads and writes only the control=1 half)."""
    S = (1 << n) * elem_bytes
    n_cnot = sum(len(range(l % 2, n - 1, 2)) for l in range(layers))
    return layers * 2 * n * 2 * S + n_cnot * S


def random_3regular_graph(n: int, st: Stream, max_tries: int = 10000) -> list:
    """Uniform-ish random simple 3-regular graph: shuffle the 3n edge stubs with
    Fisher-Yates (one draw per swap, j = floor(u*(i+1))), pair stubs 2k/2k+1,
    reject on self-loops or repeated edges.  n must be even."""
    if n % 2 or n < 4:
        raise ValueError("3-regular graphs need an even n >= 4")
    for _ in range(max_tries):
        stubs = np.repeat(np.arange(n), 3)
        u = st.take(len(stubs) - 1)
        for k, i in enumerate(range(len(stubs) - 1, 0, -1)):
            j = min(int(u[k] * (i + 1)), i)
            stubs[i], stubs[j] = stubs[j], stubs[i]
        edges = set()
        ok = True
        for k in range(0, len(stubs), 2):
            a, b = int(stubs[k]), int(stubs[k + 1])
            if a == b:
                ok = False
                break
            e = (min(a, b), max(a, b))
            if e in edges:
                ok = False
                break
            edges.add(e)
        if ok:
            return sorted(edges)
    raise RuntimeError("no simple 3-regular graph found")


def qaoa_instances(count: int, seed: int, n_values=tuple(range(12, 25, 2)), p: int = 4):
    """Batched QAOA MaxCut instances: n uniform over n_values, a random 3-regular
    graph with unit weights, gamma_l ~ U[0, pi), beta_l ~ U[0, pi/2).
    Returns a list of dicts {n, edges [(i, j, w)], gammas, betas}."""
    size_st = Stream(seed, 3)
    graph_st = Stream(seed, 2)
    out = []
    for _ in range(count):
        n = int(n_values[size_st.randint(len(n_values))])
        e = random_3regular_graph(n, graph_st)
        ang = size_st.take(2 * p)
        out.append(dict(n=n, edges=[(i, j, 1.0) for i, j in e],
                        gammas=ang[:p] * math.pi, betas=ang[p:] * (math.pi / 2)))
    return out


def pauli_hamiltonian(n: int, terms: int, seed: int):
    """Random Pauli strings: each qubit I/X/Y/Z with probability 1/4 each
    (op = floor(4u)), coefficients ~ N(0, 1).  Returns (coeffs, [ops...]) with
    ops as [(qubit, op)] lists of the non-identity factors."""
    st = Stream(seed, 4)
    codes = np.minimum((st.take(terms * n) * 4).astype(np.int64), 3).reshape(terms, n)
    coeffs = st.normal(terms)
    strings = [[(q, int(c)) for q, c in enumerate(row) if c != 0] for row in codes]
    return coeffs, strings


def hea_ry_cz(n: int, depth: int, params) -> list:
    """Hardware-efficient ansatz: per layer Ry(params) on every qubit, then a CZ
    ladder CZ(q, q+1), q = 0..n-2.  n*depth parameters."""
    params = np.asarray(params, dtype=np.float64)
    gates = []
    k = 0
    for _ in range(depth):
        for q in range(n):
            gates.append((int(GateKind.Ry), q, 0, float(params[k])))
            k += 1
        for q in range(n - 1):
            gates.append((int(GateKind.CZ), q, q + 1, 0.0))
    return gates


def vqe_parameter_sets(count: int, nparams: int, seed: int) -> np.ndarray:
    """count x nparams angles ~ U[-pi, pi)."""
    st = Stream(seed, 5)
    return st.take(count * nparams).reshape(count, nparams) * TWO_PI - math.pi
