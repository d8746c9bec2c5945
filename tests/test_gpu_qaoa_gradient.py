"""Exact QAOA gradients of the batched engine's adjoint pass (needs a GPU).

The oracle's evaluate_qaoa_cost restatement (qaoa.rs:179-201, gate-by-gate
circuit of qaoa.rs:125-153 on an f64 state) is differentiated by central
differences with h = 1e-5 (truncation and rounding both below 1e-8 here); the
device gradients must agree within 1e-7 for f64 states and 2e-4 x |E| for
f32 states.  The shift rule of run_qaoa (qaoa.rs:275-297) is checked to vanish
for unit edge weights, which is why the optimizer defaults to the adjoint.
"""
import math

import numpy as np
import pytest

import oracle
from ruqu_b200 import rng, workloads
from ruqu_b200.batch import QaoaBatch

pytestmark = pytest.mark.gpu


def _graphs(sizes, seed):
    st = rng.Stream(seed, 2)
    r = np.random.default_rng(seed)
    out = []
    for n in sizes:
        if n % 2 == 0 and n >= 4:
            out.append((n, workloads.random_3regular_graph(n, st)))
        else:   # odd n: random simple graph with ~1.5 n edges
            pairs = [(i, j) for i in range(n) for j in range(i + 1, n)]
            pick = r.choice(len(pairs), size=min(len(pairs), (3 * n) // 2), replace=False)
            out.append((n, [pairs[k] for k in sorted(pick)]))
    return out


def _fd_gradient(n, edges, g, b, h=1e-5):
    ew = [(u, v, 1.0) for u, v in edges]
    th = np.concatenate([g, b]).astype(np.float64)
    p = len(g)
    out = np.zeros(2 * p)
    for k in range(2 * p):
        tp, tm = th.copy(), th.copy()
        tp[k] += h
        tm[k] -= h
        out[k] = (oracle.qaoa_cost(n, ew, tp[:p], tp[p:]) - oracle.qaoa_cost(n, ew, tm[:p], tm[p:])) / (2 * h)
    return out, oracle.qaoa_cost(n, ew, th[:p], th[p:])


@pytest.mark.parametrize("prec,sizes", [("f64", [6, 7, 8, 10, 12, 13, 14]), ("f32", [7, 8, 12, 14, 15, 16])])
@pytest.mark.parametrize("p", [1, 3])
def test_adjoint_gradients_match_finite_differences(prec, sizes, p):
    graphs = _graphs(sizes, 40 + p)
    r = np.random.default_rng(p + 17)
    gam = r.uniform(0, math.pi, size=(len(graphs), p))
    bet = r.uniform(0, math.pi / 2, size=(len(graphs), p))
    qb = QaoaBatch(graphs, p, prec)
    e, grad = qb.gradient(gam, bet)
    for k, (n, ed) in enumerate(graphs):
        want, we = _fd_gradient(n, ed, gam[k], bet[k])
        tol = 1e-7 if prec == "f64" else 2e-4 * max(1.0, abs(we))
        assert abs(e[k] - we) < (1e-10 if prec == "f64" else 1e-5 * len(ed)), (n, e[k], we)
        assert np.max(np.abs(grad[k] - want)) < tol, (n, grad[k], want)


def test_gradient_is_independent_of_the_batch():
    graphs = _graphs([12, 14, 14, 16], 3)
    r = np.random.default_rng(5)
    gam = r.uniform(0, math.pi, size=(4, 4))
    bet = r.uniform(0, math.pi / 2, size=(4, 4))
    _, ga = QaoaBatch(graphs, 4, "f32").gradient(gam, bet)
    for k in range(4):
        _, gs = QaoaBatch([graphs[k]], 4, "f32").gradient(gam[k:k + 1], bet[k:k + 1])
        assert np.array_equal(ga[k], gs[0])
    small = QaoaBatch(graphs, 4, "f32")
    small.set_state_budget(1 << 20)      # one circuit's psi and lambda per wave
    _, gw = small.gradient(gam, bet)
    assert np.array_equal(ga, gw)


def test_reference_shift_rule_vanishes_for_unit_weights():
    graphs = _graphs([8, 10, 11], 9)
    p = 2
    r = np.random.default_rng(2)
    gam = r.uniform(0, math.pi, size=(3, p))
    bet = r.uniform(0, math.pi / 2, size=(3, p))
    sets_g, sets_b = [], []
    for k in range(3):
        th = np.concatenate([gam[k], bet[k]])
        rows = [th]
        for j in range(2 * p):
            for d in (math.pi / 2, -math.pi / 2):
                t = th.copy()
                t[j] += d
                rows.append(t)
        rows = np.array(rows)
        sets_g.append(rows[:, :p])
        sets_b.append(rows[:, p:])
    qb = QaoaBatch(graphs, p, "f64")
    e = qb.run(np.array(sets_g), np.array(sets_b))["energies"]
    shift = (e[:, 1::2] - e[:, 2::2]) / 2
    assert np.max(np.abs(shift)) < 1e-12
    _, grad = qb.gradient(gam, bet)
    assert np.max(np.abs(grad)) > 1e-3
