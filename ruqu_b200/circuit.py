"""Fluent circuit builder (crates/ruqu-core/src/circuit.rs:8-185)."""
from __future__ import annotations

import ctypes as C

from ._capi import RqGate
from .gate import Gate, GateKind


def gates_to_array(gates) -> C.Array:
    """Pack Gate objects (or (kind, q0, q1, angle[, m8]) tuples) into an rq_gate array."""
    arr = (RqGate * max(1, len(gates)))()
    for k, g in enumerate(gates):
        t = g.to_tuple() if isinstance(g, Gate) else g
        arr[k].kind = int(t[0])
        arr[k].q0 = int(t[1])
        arr[k].q1 = int(t[2]) if len(t) > 2 else 0
        arr[k].angle = float(t[3]) if len(t) > 3 else 0.0
        if len(t) > 4 and t[4] is not None:
            for i in range(8):
                arr[k].m[i] = float(t[4][i])
    return arr


class QuantumCircuit:
    """Ordered gate list on a qubit register."""

    def __init__(self, num_qubits: int):
        self._n = int(num_qubits)
        self._gates: list = []
        self._packed = None

    # ---- single-qubit gates (circuit.rs:26-69) ----
    def _push(self, g: Gate) -> "QuantumCircuit":
        self._gates.append(g)
        self._packed = None
        return self

    def h(self, q): return self._push(Gate.H(q))
    def x(self, q): return self._push(Gate.X(q))
    def y(self, q): return self._push(Gate.Y(q))
    def z(self, q): return self._push(Gate.Z(q))
    def s(self, q): return self._push(Gate.S(q))
    def t(self, q): return self._push(Gate.T(q))
    def rx(self, q, angle): return self._push(Gate.Rx(q, angle))
    def ry(self, q, angle): return self._push(Gate.Ry(q, angle))
    def rz(self, q, angle): return self._push(Gate.Rz(q, angle))
    def phase(self, q, angle): return self._push(Gate.Phase(q, angle))

    # ---- two-qubit gates (circuit.rs:75-98) ----
    def cnot(self, control, target): return self._push(Gate.CNOT(control, target))
    def cz(self, q1, q2): return self._push(Gate.CZ(q1, q2))
    def swap(self, q1, q2): return self._push(Gate.SWAP(q1, q2))
    def rzz(self, q1, q2, angle): return self._push(Gate.Rzz(q1, q2, angle))

    # ---- special operations (circuit.rs:104-134) ----
    def measure(self, q): return self._push(Gate.Measure(q))

    def measure_all(self):
        for q in range(self._n):
            self._push(Gate.Measure(q))
        return self

    def reset(self, q): return self._push(Gate.Reset(q))
    def barrier(self): return self._push(Gate.Barrier())
    def add_gate(self, gate: Gate): return self._push(gate)

    # ---- accessors (circuit.rs:140-184) ----
    def gates(self) -> list:
        return self._gates

    def num_qubits(self) -> int:
        return self._n

    def gate_count(self) -> int:
        return len(self._gates)

    def depth(self) -> int:
        """Longest qubit-dependency path; a Barrier levels all qubits (circuit.rs:156-184)."""
        qd = [0] * self._n
        for g in self._gates:
            if g.kind == GateKind.Barrier:
                mx = max(qd) if qd else 0
                qd = [mx] * self._n
                continue
            qs = g.qubits()
            if not qs:
                continue
            mx = max(qd[q] if q < self._n else 0 for q in qs)
            for q in qs:
                if q < self._n:
                    qd[q] = mx + 1
        return max(qd) if qd else 0

    def packed(self) -> C.Array:
        """The rq_gate array handed to the C ABI (cached until the circuit changes)."""
        if self._packed is None:
            self._packed = gates_to_array(self._gates)
        return self._packed
