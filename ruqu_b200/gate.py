"""Gate definitions and matrices (crates/ruqu-core/src/gate.rs:8-198).

``Gate`` mirrors the reference enum: construct with ``Gate.H(q)``,
``Gate.CNOT(c, t)``, ``Gate.Rx(q, theta)`` ...  ``kind`` codes are the
rq_gate_kind values of include/ruqu_cuda.h.
"""
from __future__ import annotations

import enum
import math

import numpy as np


class GateKind(enum.IntEnum):
    H = 0
    X = 1
    Y = 2
    Z = 3
    S = 4
    Sdg = 5
    T = 6
    Tdg = 7
    Rx = 8
    Ry = 9
    Rz = 10
    Phase = 11
    CNOT = 12
    CZ = 13
    SWAP = 14
    Rzz = 15
    Measure = 16
    Reset = 17
    Barrier = 18
    Unitary1Q = 19


_TWO_QUBIT = {GateKind.CNOT, GateKind.CZ, GateKind.SWAP, GateKind.Rzz}
_ANGLED = {GateKind.Rx, GateKind.Ry, GateKind.Rz, GateKind.Phase, GateKind.Rzz}
FRAC_1_SQRT_2 = 0.7071067811865476


class Gate:
    __slots__ = ("kind", "q0", "q1", "angle", "matrix")

    def __init__(self, kind: GateKind, q0: int = 0, q1: int = 0, angle: float = 0.0, matrix=None):
        self.kind = GateKind(kind)
        self.q0 = int(q0)
        self.q1 = int(q1)
        self.angle = float(angle)
        self.matrix = None if matrix is None else np.asarray(matrix, dtype=np.complex128).reshape(2, 2)

    # ---- constructors named like the reference variants ----
    @classmethod
    def H(cls, q): return cls(GateKind.H, q)
    @classmethod
    def X(cls, q): return cls(GateKind.X, q)
    @classmethod
    def Y(cls, q): return cls(GateKind.Y, q)
    @classmethod
    def Z(cls, q): return cls(GateKind.Z, q)
    @classmethod
    def S(cls, q): return cls(GateKind.S, q)
    @classmethod
    def Sdg(cls, q): return cls(GateKind.Sdg, q)
    @classmethod
    def T(cls, q): return cls(GateKind.T, q)
    @classmethod
    def Tdg(cls, q): return cls(GateKind.Tdg, q)
    @classmethod
    def Rx(cls, q, theta): return cls(GateKind.Rx, q, angle=theta)
    @classmethod
    def Ry(cls, q, theta): return cls(GateKind.Ry, q, angle=theta)
    @classmethod
    def Rz(cls, q, theta): return cls(GateKind.Rz, q, angle=theta)
    @classmethod
    def Phase(cls, q, theta): return cls(GateKind.Phase, q, angle=theta)
    @classmethod
    def CNOT(cls, c, t): return cls(GateKind.CNOT, c, t)
    @classmethod
    def CZ(cls, a, b): return cls(GateKind.CZ, a, b)
    @classmethod
    def SWAP(cls, a, b): return cls(GateKind.SWAP, a, b)
    @classmethod
    def Rzz(cls, a, b, theta): return cls(GateKind.Rzz, a, b, theta)
    @classmethod
    def Measure(cls, q): return cls(GateKind.Measure, q)
    @classmethod
    def Reset(cls, q): return cls(GateKind.Reset, q)
    @classmethod
    def Barrier(cls): return cls(GateKind.Barrier)
    @classmethod
    def Unitary1Q(cls, q, m): return cls(GateKind.Unitary1Q, q, matrix=m)

    def __repr__(self):
        k = self.kind.name
        if self.kind == GateKind.Barrier:
            return "Barrier"
        args = [str(q) for q in self.qubits()]
        if self.kind in _ANGLED:
            args.append(repr(self.angle))
        return f"{k}({', '.join(args)})"

    def qubits(self) -> list:
        """gate.rs:40-63."""
        if self.kind == GateKind.Barrier:
            return []
        if self.kind in _TWO_QUBIT:
            return [self.q0, self.q1]
        return [self.q0]

    def is_non_unitary(self) -> bool:
        """gate.rs:66-68."""
        return self.kind in (GateKind.Measure, GateKind.Reset, GateKind.Barrier)

    def matrix_1q(self):
        """2x2 matrix of a single-qubit gate, else None (gate.rs:72-146)."""
        k = self.kind
        c0, c1, ci = 0j, 1 + 0j, 1j
        s = FRAC_1_SQRT_2
        if k == GateKind.H:
            m = [[s, s], [s, -s]]
        elif k == GateKind.X:
            m = [[c0, c1], [c1, c0]]
        elif k == GateKind.Y:
            m = [[c0, -ci], [ci, c0]]
        elif k == GateKind.Z:
            m = [[c1, c0], [c0, -c1]]
        elif k == GateKind.S:
            m = [[c1, c0], [c0, ci]]
        elif k == GateKind.Sdg:
            m = [[c1, c0], [c0, -ci]]
        elif k == GateKind.T:
            m = [[c1, c0], [c0, complex(s, s)]]
        elif k == GateKind.Tdg:
            m = [[c1, c0], [c0, complex(s, -s)]]
        elif k == GateKind.Rx:
            h = self.angle / 2.0
            c, sn = complex(math.cos(h), 0.0), complex(0.0, -math.sin(h))
            m = [[c, sn], [sn, c]]
        elif k == GateKind.Ry:
            h = self.angle / 2.0
            m = [[math.cos(h), -math.sin(h)], [math.sin(h), math.cos(h)]]
        elif k == GateKind.Rz:
            h = self.angle / 2.0
            m = [[complex(math.cos(-h), math.sin(-h)), c0], [c0, complex(math.cos(h), math.sin(h))]]
        elif k == GateKind.Phase:
            m = [[c1, c0], [c0, complex(math.cos(self.angle), math.sin(self.angle))]]
        elif k == GateKind.Unitary1Q:
            return self.matrix.copy()
        else:
            return None
        return np.array(m, dtype=np.complex128)

    def matrix_2q(self):
        """4x4 matrix of a two-qubit gate, index = q1_bit*2 + q2_bit (gate.rs:148-198)."""
        k = self.kind
        m = np.zeros((4, 4), dtype=np.complex128)
        if k == GateKind.CNOT:
            m[0, 0] = m[1, 1] = m[2, 3] = m[3, 2] = 1
        elif k == GateKind.CZ:
            m[0, 0] = m[1, 1] = m[2, 2] = 1
            m[3, 3] = -1
        elif k == GateKind.SWAP:
            m[0, 0] = m[1, 2] = m[2, 1] = m[3, 3] = 1
        elif k == GateKind.Rzz:
            h = self.angle / 2.0
            en = complex(math.cos(-h), math.sin(-h))
            ep = complex(math.cos(h), math.sin(h))
            m[0, 0], m[1, 1], m[2, 2], m[3, 3] = en, ep, ep, en
        else:
            return None
        return m

    def to_tuple(self):
        """(kind, q0, q1, angle, m8-or-None): the plain form the C ABI struct is filled from."""
        m8 = None
        if self.kind == GateKind.Unitary1Q:
            m8 = [v for c in self.matrix.reshape(-1) for v in (c.real, c.imag)]
        return (int(self.kind), self.q0, self.q1, self.angle, m8)
