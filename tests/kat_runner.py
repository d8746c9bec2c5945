"""Runs the reference known-answer cases (tests/golden/reference_kats.py) on a backend.

A backend is any object with: apply(list of (kind,q0,q1,angle)), reset(q),
probs(), amps(), expect(ops), ham(list of (coeff, ops)), prob_qubit(q).
"""
import numpy as np


def run_case(backend, case, eps):
    for st in case["steps"]:
        if st[0] == "g":
            backend.apply([st[1:]])
        elif st[0] == "reset":
            backend.reset(st[1])
    for chk in case["checks"]:
        kind = chk[0]
        where = f'{case["name"]} ({case["ref"]}) {chk}'
        if kind == "prob":
            assert abs(backend.probs()[chk[1]] - chk[2]) < eps, where
        elif kind == "probs_zero_except":
            p = backend.probs()
            for i in range(len(p)):
                if i not in chk[1]:
                    assert abs(p[i]) < eps, where
        elif kind == "amp":
            a = backend.amps()[chk[1]]
            assert abs(a.real - chk[2]) < eps, where
            if chk[3] is not None:
                assert abs(a.imag - chk[3]) < eps, where
        elif kind == "expect":
            assert abs(backend.expect(chk[1]) - chk[2]) < eps, where
        elif kind == "ham":
            assert abs(backend.ham(chk[1]) - chk[2]) < eps, where
        elif kind == "prob_qubit":
            assert abs(backend.prob_qubit(chk[1]) - chk[2]) < eps, where
        elif kind == "total":
            assert abs(float(np.sum(backend.probs())) - chk[1]) < eps, where
        else:
            raise AssertionError(f"unknown check {kind}")


class OracleBackend:
    def __init__(self, n, precision, seed=42):
        import oracle
        self.s = oracle.OracleState(n, precision, seed)

    def apply(self, gates):
        return self.s.apply(gates)

    def reset(self, q):
        self.s.reset_qubit(q)

    def probs(self):
        return self.s.probabilities()

    def amps(self):
        return self.s.amplitudes()

    def expect(self, ops):
        return self.s.expectation(ops)

    def ham(self, terms):
        return self.s.expectation_hamiltonian([c for c, _ in terms], [o for _, o in terms])

    def prob_qubit(self, q):
        return self.s.probability_of_qubit(q)


class GpuBackend:
    def __init__(self, n, precision, seed=42, mode=0):
        from ruqu_b200 import QuantumState
        self.s = QuantumState(n, seed, "f32" if precision == 0 else "f64")
        self.mode = mode

    def apply(self, gates):
        return self.s.apply_gates(gates, self.mode)

    def reset(self, q):
        self.s.reset_qubit(q)

    def probs(self):
        return self.s.probabilities()

    def amps(self):
        return self.s.state_vector()

    def expect(self, ops):
        return self.s.expectation_value(ops)

    def ham(self, terms):
        from ruqu_b200 import Hamiltonian, PauliString
        return self.s.expectation_hamiltonian(Hamiltonian([(c, PauliString(o)) for c, o in terms], 0))

    def prob_qubit(self, q):
        return self.s.probability_of_qubit(q)
