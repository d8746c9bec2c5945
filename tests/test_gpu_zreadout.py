"""Single-qubit Z expectations through the one-pass read-out kernel (needs a GPU).

rq_state_expectation_batch sends every string that is the identity or a single
Z (after the reference's mask reduction, state.rs:362-408) through one pass
for up to 32 of them; the others keep the grouped Pauli passes.  Checked
against the oracle's per-string expectations: 1e-10 absolute for f64 states,
1e-5 for f32, including mixed lists (slot mapping) and more than 32 Z strings
(two passes).
"""
import numpy as np
import pytest

import oracle
from ruqu_b200 import QuantumState, workloads

pytestmark = pytest.mark.gpu

PREC = {"f64": oracle.RQ_F64, "f32": oracle.RQ_F32}
TOL = {"f64": 1e-10, "f32": 1e-5}


def _states(n, prec, seed):
    gates = workloads.random_layer_circuit(n, 3, seed)
    g = QuantumState(n, 0, prec)
    g.apply_gates(gates)
    o = oracle.OracleState(n, PREC[prec], 0)
    o.apply(gates)
    return g, o


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n", [5, 7, 12, 20])
def test_all_z_and_identity(prec, n):
    g, o = _states(n, prec, n)
    strings = [[(q, 3)] for q in range(n)] + [[]]
    got = g.expectation_values(strings)
    want = np.array([o.expectation(s) for s in strings])
    assert np.max(np.abs(got - want)) < TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_mixed_lists_and_two_passes(prec):
    n = 14
    g, o = _states(n, prec, 3)
    r = np.random.default_rng(4)
    strings = []
    for k in range(80):
        kind = k % 4
        if kind == 0:
            strings.append([(int(r.integers(0, n)), 3)])                    # single Z
        elif kind == 1:
            strings.append([(int(r.integers(0, n)), int(r.integers(1, 3)))])  # X or Y
        elif kind == 2:
            a, b = r.choice(n, 2, replace=False)
            strings.append([(int(a), 3), (int(b), 3)])                       # ZZ
        else:
            q = int(r.integers(0, n))
            strings.append([(q, 2), (q, 2)])                                 # Y.Y on one qubit: -I... as reduced
    strings += [[(q, 3)] for q in range(n)] * 3                              # > 32 single-Z strings
    got = g.expectation_values(strings)
    want = np.array([o.expectation(s) for s in strings])
    assert np.max(np.abs(got - want)) < TOL[prec]
