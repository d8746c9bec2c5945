"""Kraus operator sets of single-qubit noise channels (crates/ruqu-core/src/noise.rs:151-280).

Pure host code (numpy; the CUDA library is not loaded).  Each constructor returns a
``(k, 2, 2)`` complex128 array whose entries follow the reference constructor's
formula and clamping exactly.  ``QuantumState.apply_kraus`` applies such a set to one
qubit of a device state as a quantum-trajectory step (``rq_state_apply_kraus``).
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["depolarizing_kraus", "amplitude_damping_kraus", "phase_damping_kraus",
           "thermal_relaxation_kraus", "completeness_error"]


def depolarizing_kraus(p: float) -> np.ndarray:
    """sqrt(1-p) I, sqrt(p/3) X, sqrt(p/3) Y, sqrt(p/3) Z (noise.rs:166-188), both
    square roots of arguments clamped at 0."""
    s0 = math.sqrt(max(1.0 - p, 0.0))
    sp = math.sqrt(max(p / 3.0, 0.0))
    return np.array([
        [[s0, 0], [0, s0]],
        [[0, sp], [sp, 0]],
        [[0, -1j * sp], [1j * sp, 0]],
        [[sp, 0], [0, -sp]],
    ], dtype=np.complex128)


def amplitude_damping_kraus(gamma: float) -> np.ndarray:
    """[[1,0],[0,sqrt(1-gamma)]] and [[0,sqrt(gamma)],[0,0]] (noise.rs:197-208); gamma is
    clamped to [0, 1] under the first root and 1-gamma at 0 under the second."""
    sg = math.sqrt(min(max(gamma, 0.0), 1.0))
    s1g = math.sqrt(max(1.0 - gamma, 0.0))
    return np.array([[[1, 0], [0, s1g]], [[0, sg], [0, 0]]], dtype=np.complex128)


def phase_damping_kraus(lam: float) -> np.ndarray:
    """[[1,0],[0,sqrt(1-lambda)]] and [[0,0],[0,sqrt(lambda)]] (noise.rs:217-228)."""
    sl = math.sqrt(min(max(lam, 0.0), 1.0))
    s1l = math.sqrt(max(1.0 - lam, 0.0))
    return np.array([[[1, 0], [0, s1l]], [[0, 0], [0, sl]]], dtype=np.complex128)


def thermal_relaxation_kraus(t1: float, t2: float, gate_time: float) -> np.ndarray:
    """Amplitude damping with gamma = 1 - exp(-t/T1) composed with phase damping of the
    residual dephasing rate 1/T2' - 1/(2 T1), T2' = min(T2, 2 T1); the four products
    K_ad K_pd in the order (ad, pd) of noise.rs:245-286.  The identity alone when the
    gate time or T1 is not positive (noise.rs:247-249)."""
    if gate_time <= 0.0 or t1 <= 0.0:
        return np.eye(2, dtype=np.complex128)[None]
    gamma = 1.0 - math.exp(-gate_time / t1)
    t2_eff = min(t2, 2.0 * t1)
    inv_t_phi = (1.0 / t2_eff) - (1.0 / (2.0 * t1)) if t2_eff > 0.0 else 0.0
    lam = 1.0 - math.exp(-gate_time * inv_t_phi) if inv_t_phi > 0.0 else 0.0
    ad = amplitude_damping_kraus(gamma)
    pd = phase_damping_kraus(lam)
    return np.array([a @ b for a in ad for b in pd], dtype=np.complex128)


def completeness_error(ops) -> float:
    """max |sum_k K_k^dagger K_k - I|: 0 for a trace-preserving set (the property the
    reference's tests assert, noise.rs:643-690)."""
    k = np.asarray(ops, dtype=np.complex128).reshape(-1, 2, 2)
    s = np.einsum("kji,kjl->il", k.conj(), k)
    return float(np.abs(s - np.eye(2)).max())
