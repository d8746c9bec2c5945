"""Exact VQE gradients by the adjoint pass vs the parameter-shift rule (needs a GPU).

For Ry(theta) = exp(-i theta Y / 2) the shift rule of run_vqe (vqe.rs:186-198),
(E(theta + pi/2) - E(theta - pi/2)) / 2, is the exact derivative, so the adjoint
gradients (RQ_VQE_GRAD_ADJOINT) must equal the device's shift gradients and the
oracle's shift differences up to rounding: 1e-10 absolute for f64 states, 1e-5
relative to sum |coeff| for f32 states.
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


def _hamiltonian(n, terms, seed):
    coeffs, strings = workloads.pauli_hamiltonian(n, terms, seed)
    # repeated qubits (Y0 Y0; X1 X1 Z3), an identity string and an anti-Hermitian
    # product (X0 Z0, no real expectation)
    strings = strings + [[(0, 2), (0, 2)], [(1, 1), (1, 1), (3, 3)], [], [(0, 1), (0, 3)]]
    coeffs = np.concatenate([coeffs, [0.3, -0.7, 1.1, 0.9]])
    return coeffs, strings


@pytest.mark.parametrize("prec,n,depth", [("f64", 8, 3), ("f32", 9, 2), ("f64", 6, 2), ("f32", 7, 3)])
def test_adjoint_equals_shift_rule(prec, n, depth):
    coeffs, strings = _hamiltonian(n, 24, 5)
    P = n * depth
    params = np.random.default_rng(2).uniform(-math.pi, math.pi, size=(3, P))
    vb = VqeBatch(n, depth, coeffs, strings, prec)
    e_s, g_s = vb.run(params, gradient="shift")
    e_a, g_a = vb.run(params, gradient="adjoint")
    scale = float(np.sum(np.abs(coeffs)))
    tol = 1e-10 if prec == "f64" else 1e-5 * scale
    assert np.array_equal(e_a, e_s)                      # the same forward pass
    assert np.max(np.abs(g_a - g_s)) < tol, np.max(np.abs(g_a - g_s))
    for k in range(0, P, max(1, P // 5)):
        pp, pm = params[1].copy(), params[1].copy()
        pp[k] += math.pi / 2
        pm[k] -= math.pi / 2
        want = (_energy(n, depth, pp, coeffs, strings) - _energy(n, depth, pm, coeffs, strings)) / 2
        assert abs(g_a[1, k] - want) < tol, (k, g_a[1, k], want)


def test_adjoint_16q_200_strings():
    """The batched-VQE shape: 16 qubits, 200 random strings (seed 3), depth 8 (128
    parameters), f32 states, several tiles per state in the adjoint program."""
    n, depth = 16, 8
    coeffs, strings = workloads.pauli_hamiltonian(n, 200, 3)
    params = workloads.vqe_parameter_sets(4, n * depth, 4)
    vb = VqeBatch(n, depth, coeffs, strings, "f32")
    e_s, g_s = vb.run(params, gradient="shift")
    e_a, g_a = vb.run(params, gradient="adjoint")
    scale = float(np.sum(np.abs(coeffs)))
    assert np.array_equal(e_a, e_s)
    assert np.max(np.abs(g_a - g_s)) < 1e-5 * scale, np.max(np.abs(g_a - g_s))
    # deterministic: a second run gives the same bits
    e_b, g_b = vb.run(params, gradient="adjoint")
    assert np.array_equal(g_a, g_b) and np.array_equal(e_a, e_b)


def test_adjoint_wave_boundaries_f64():
    """More parameter sets than one wave holds (20-qubit f64 states of 16 MiB: six per
    96 MiB wave): every set's gradient must match its own single-set run."""
    n, depth = 20, 1
    coeffs, strings = _hamiltonian(n, 16, 7)
    params = np.random.default_rng(4).uniform(-math.pi, math.pi, size=(8, n * depth))
    vb = VqeBatch(n, depth, coeffs, strings, "f64")
    e, g = vb.run(params, gradient="adjoint")
    for s in (0, 5, 6, 7):
        e1, g1 = vb.run(params[s:s + 1], gradient="adjoint")
        assert abs(e1[0] - e[s]) < 1e-12
        assert np.max(np.abs(g1[0] - g[s])) < 1e-10


def test_empty_hamiltonian_gives_zero_gradient():
    vb = VqeBatch(7, 2, np.zeros(0), [], "f32")
    e, g = vb.run(np.full((2, 14), 0.3), gradient="adjoint")
    assert np.all(e == 0.0) and np.all(g == 0.0)
