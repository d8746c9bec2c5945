"""Batched VQE engine vs the oracle (needs a GPU).

Energies: the oracle's expectation_hamiltonian (state.rs:403-408) on the same
Ry + CZ-ladder ansatz run gate by gate; tolerance 1e-10 absolute for f64
states, 1e-5 relative (to sum |coeff|) for f32 states.  Gradients: the
parameter-shift difference of oracle energies (vqe.rs:186-198).
"""
import math

import numpy as np
import pytest

import oracle
from ruqu_b200 import workloads
from ruqu_b200.batch import VqeBatch

pytestmark = pytest.mark.gpu


def _energy(n, depth, params, coeffs, strings):
    return oracle.circuit_energy(n, workloads.hea_ry_cz(n, depth, params), coeffs, strings)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_vqe_batch_energies_and_gradients(prec):
    n, depth = (8, 3) if prec == "f64" else (9, 2)
    coeffs, strings = workloads.pauli_hamiltonian(n, 24, 5)
    strings = strings + [[(0, 2), (0, 2)], [(1, 1), (1, 1), (3, 3)], []]   # repeated qubits, identity
    coeffs = np.concatenate([coeffs, [0.3, -0.7, 1.1]])
    P = n * depth
    r = np.random.default_rng(1)
    params = r.uniform(-math.pi, math.pi, size=(3, P))
    vb = VqeBatch(n, depth, coeffs, strings, prec)
    e, g = vb.run(params, gradient=True)
    scale = float(np.sum(np.abs(coeffs)))
    tol = 1e-10 if prec == "f64" else 1e-5 * scale
    for s in range(3):
        assert abs(e[s] - _energy(n, depth, params[s], coeffs, strings)) < tol
        for k in range(0, P, max(1, P // 6)):
            pp, pm = params[s].copy(), params[s].copy()
            pp[k] += math.pi / 2
            pm[k] -= math.pi / 2
            want = (_energy(n, depth, pp, coeffs, strings) - _energy(n, depth, pm, coeffs, strings)) / 2
            assert abs(g[s, k] - want) < tol, (s, k, g[s, k], want)
    e2 = vb.run(params)
    assert np.max(np.abs(e2 - e)) == 0.0


def test_vqe_batch_config_shape_16q():
    """16 qubits, 200 random Pauli strings (seed 3), depth 8 Ry + CZ ladder, f32 states."""
    n, depth = 16, 8
    coeffs, strings = workloads.pauli_hamiltonian(n, 200, 3)
    params = workloads.vqe_parameter_sets(2, n * depth, 4)
    vb = VqeBatch(n, depth, coeffs, strings, "f32")
    e, g = vb.run(params, gradient=True)
    scale = float(np.sum(np.abs(coeffs)))
    for s in range(2):
        want = _energy(n, depth, params[s], coeffs, strings)
        assert abs(e[s] - want) < 1e-5 * scale, (e[s], want)
    k = 37
    pp, pm = params[0].copy(), params[0].copy()
    pp[k] += math.pi / 2
    pm[k] -= math.pi / 2
    want = (_energy(n, depth, pp, coeffs, strings) - _energy(n, depth, pm, coeffs, strings)) / 2
    assert abs(g[0, k] - want) < 1e-5 * scale


def test_vqe_batch_f64_two_energy_tiles():
    """f64 states above 12 qubits: the energy kernel pairs 2^12-amplitude tiles."""
    n, depth = 14, 2
    coeffs, strings = workloads.pauli_hamiltonian(n, 12, 8)
    params = workloads.vqe_parameter_sets(2, n * depth, 9)
    vb = VqeBatch(n, depth, coeffs, strings, "f64")
    e = vb.run(params)
    for s in range(2):
        want = _energy(n, depth, params[s], coeffs, strings)
        assert abs(e[s] - want) < 1e-10, (e[s], want)


@pytest.mark.parametrize("gradient", [False, "shift", "adjoint"])
def test_vqe_runs_replay_one_graph_with_identical_results(gradient):
    """rq_vqe_batch_run as a CUDA graph: results equal a batch
    that never uses graphs, for new parameters every run; the first run of a shape is plain,
    later ones launch the captured graph."""
    n, depth = 12, 3
    coeffs, strings = workloads.pauli_hamiltonian(n, 40, 7)
    P = n * depth
    r = np.random.default_rng(8)
    a = VqeBatch(n, depth, coeffs, strings, "f32")
    b = VqeBatch(n, depth, coeffs, strings, "f32")
    b.set_graphs(False)
    flags = []
    for it in range(3):
        params = r.uniform(-math.pi, math.pi, size=(5, P))
        x = a.run(params, gradient=gradient)
        flags.append(a.last_graph()["replayed"])
        y = b.run(params, gradient=gradient)
        if gradient:
            assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
        else:
            assert np.array_equal(x, y)
    assert flags == [False, True, True]
