"""QAOA optimizer on the device and the learned warm start (needs a GPU).

The device Adam loop (exact adjoint gradients) is checked step for step
against the same Adam written in numpy over central differences of the
oracle's evaluate_qaoa_cost (qaoa.rs:179-201); the warm start is checked
end to end on small graphs: training reduces the loss and warm-started
instances reach the plain optimizer's energy in fewer steps.
"""

import numpy as np
import pytest

import oracle
from ruqu_b200 import rng, workloads
from ruqu_b200.batch import QaoaBatch
from ruqu_b200.warmstart import WarmStart, linear_ramp

pytestmark = pytest.mark.gpu


def _graphs(count, sizes, seed):
    st = rng.Stream(seed, 2)
    r = np.random.default_rng(seed)
    return [(int(n), workloads.random_3regular_graph(int(n), st)) for n in r.choice(sizes, size=count)]


def _host_adam(n, edges, g, b, steps, lr, h=1e-5):
    """Adam on central-difference gradients of the oracle's energy."""
    p = len(g)
    th = np.concatenate([g, b]).astype(np.float64)
    m = np.zeros_like(th)
    v = np.zeros_like(th)
    ew = [(u, w, 1.0) for u, w in edges]
    for t in range(steps):
        grad = np.zeros_like(th)
        for k in range(2 * p):
            tp, tm = th.copy(), th.copy()
            tp[k] += h
            tm[k] -= h
            grad[k] = (oracle.qaoa_cost(n, ew, tp[:p], tp[p:]) - oracle.qaoa_cost(n, ew, tm[:p], tm[p:])) / (2 * h)
        m = 0.9 * m + 0.1 * grad
        v = 0.999 * v + 0.001 * grad * grad
        th += lr * (m / (1 - 0.9 ** (t + 1))) / (np.sqrt(v / (1 - 0.999 ** (t + 1))) + 1e-8)
    return th[:p], th[p:], oracle.qaoa_cost(n, ew, th[:p], th[p:])


def test_device_adam_matches_host_adam():
    graphs = _graphs(4, [8, 10], 1)
    p, steps, lr = 2, 6, 0.05
    g0, b0 = linear_ramp(p)
    qb = QaoaBatch(graphs, p, "f64")
    g, b, e, st = qb.optimize(np.tile(g0, (4, 1)), np.tile(b0, (4, 1)), steps, lr)
    for k, (n, ed) in enumerate(graphs):
        hg, hb, he = _host_adam(n, ed, g0, b0, steps, lr)
        # exact device gradients vs 1e-5 central differences: angles agree to 1e-7
        assert np.max(np.abs(g[k] - hg)) < 1e-7 and np.max(np.abs(b[k] - hb)) < 1e-7
        assert abs(e[k] - he) < 1e-7 and st[k] == steps


def test_target_stopping():
    graphs = _graphs(6, [8, 10, 12], 2)
    p = 3
    g0, b0 = linear_ramp(p)
    G, B = np.tile(g0, (6, 1)), np.tile(b0, (6, 1))
    qb = QaoaBatch(graphs, p, "f32")
    _, _, e20, _ = qb.optimize(G, B, 20, 0.05)
    _, _, e, st = qb.optimize(G, B, 40, 0.05, target=e20, rtol=1e-5)
    assert np.all(st <= 20)
    assert np.all(e >= e20 * (1 - 1e-5) - 1e-12)


def test_finished_instances_leave_the_batch_without_changing_the_rest():
    """Instances that meet their target are dropped from the following steps' launches;
    each remaining instance follows exactly the trajectory of an uncompacted run."""
    graphs = _graphs(8, [8, 10, 12], 5)
    p = 2
    g0, b0 = linear_ramp(p)
    G, B = np.tile(g0, (8, 1)), np.tile(b0, (8, 1))
    qb = QaoaBatch(graphs, p, "f32")
    _, _, e8, _ = qb.optimize(G, B, 8, 0.05)
    tgt = np.array([e8[k] if k % 2 == 0 else len(graphs[k][1]) + 1.0 for k in range(8)])
    g, b, e, st = qb.optimize(G, B, 30, 0.05, target=tgt, rtol=1e-5)
    gf, bf, ef, _ = qb.optimize(G, B, 30, 0.05)
    for k in range(8):
        if k % 2:
            assert st[k] == 30
            assert np.array_equal(g[k], gf[k]) and np.array_equal(b[k], bf[k]) and e[k] == ef[k]
        else:
            assert st[k] <= 8
            gs, bs, es, _ = qb.optimize(G, B, int(st[k]), 0.05)
            assert np.array_equal(g[k], gs[k]) and np.array_equal(b[k], bs[k]) and e[k] == es[k]


def test_warm_start_gains_over_linear_ramp():
    """Both arms chase the same target (the energy after `steps` plain steps) with the same
    stopping rule; the learned start needs fewer steps than the linear ramp."""
    p, steps, lr = 4, 100, 0.05
    train = _graphs(768, [8, 10, 12], 3)
    held = _graphs(64, [10, 12], 4)
    g0, b0 = linear_ramp(p)
    qb = QaoaBatch(train, p, "f32")
    g, b, _, _ = qb.optimize(np.tile(g0, (len(train), 1)), np.tile(b0, (len(train), 1)), steps, lr)
    warm = WarmStart(p)
    hist = warm.fit(train, g, b, chunks=4, chunk_steps=300)
    assert len(hist) == 4 and all(np.isfinite(hist)), hist
    hb = QaoaBatch(held, p, "f32")
    G0, B0 = np.tile(g0, (len(held), 1)), np.tile(b0, (len(held), 1))
    _, _, target, _ = hb.optimize(G0, B0, steps, lr)
    _, _, e_ramp, st_ramp = hb.optimize(G0, B0, steps, lr, target=target, rtol=1e-5)
    pg, pb = warm.predict(held)
    _, _, e_warm, st_warm = hb.optimize(pg, pb, steps, 0.005, target=target, rtol=1e-5)
    assert np.mean(e_warm >= target * (1 - 1e-5)) >= 0.9
    assert np.median(st_warm) < np.median(st_ramp), (np.median(st_warm), np.median(st_ramp))


def test_step_graph_replay_equals_plain_launches(monkeypatch):
    """The optimizer replays each step as a captured CUDA graph (recaptured when finished
    instances leave); with graphs switched off the same kernels run as plain launches:
    the trajectories are identical."""
    graphs = _graphs(12, [8, 10, 12, 14], 6)
    p = 3
    g0, b0 = linear_ramp(p)
    G, B = np.tile(g0, (12, 1)), np.tile(b0, (12, 1))
    qb = QaoaBatch(graphs, p, "f32")
    _, _, e10, _ = qb.optimize(G, B, 10, 0.05)
    tgt = np.where(np.arange(12) % 3 == 0, e10, 1e9)
    ga, ba, ea, sa = qb.optimize(G, B, 25, 0.05, target=tgt, rtol=1e-5)
    monkeypatch.setenv("RUQU_NO_GRAPHS", "1")
    gb, bb, eb, sb = qb.optimize(G, B, 25, 0.05, target=tgt, rtol=1e-5)
    assert np.array_equal(ga, gb) and np.array_equal(ba, bb) and np.array_equal(ea, eb) and np.array_equal(sa, sb)


def test_preconditioned_steps_match_host_loop():
    """theta += alpha_i P_i grad, alpha_i halved when the energy fell, frozen at the target:
    the device loop against the same rule on the host over the engine's exact gradients."""
    graphs = _graphs(5, [8, 10, 12], 8)
    p, steps = 2, 6
    g0, b0 = linear_ramp(p)
    G, B = np.tile(g0, (5, 1)), np.tile(b0, (5, 1))
    r = np.random.default_rng(3)
    A = r.normal(size=(5, 2 * p, 2 * p))
    P = 0.01 * (np.einsum('kij,klj->kil', A, A) + np.eye(2 * p))
    qb = QaoaBatch(graphs, p, "f64")
    _, _, e3, _ = qb.optimize(G, B, 3, 0.05)
    target = np.where(np.arange(5) % 2 == 0, e3, 1e9)
    g, b, e, st = qb.optimize_precond(G, B, P, steps, 0.8, target=target, rtol=1e-5)
    th = np.concatenate([G, B], axis=1)
    alpha = np.full(5, 0.8)
    eprev = np.full(5, -1e300)
    done = np.zeros(5, dtype=int)
    elast = np.zeros(5)
    for t in range(steps + 1):
        en, gr = qb.gradient(th[:, :p], th[:, p:])
        for k in range(5):
            if done[k]:
                continue
            elast[k] = en[k]
            if en[k] >= target[k] * (1 - 1e-5):
                done[k] = t + 1
                continue
            if t == steps:
                continue
            if en[k] < eprev[k]:
                alpha[k] *= 0.5
            eprev[k] = en[k]
            th[k] += alpha[k] * (P[k] @ gr[k])
    assert np.max(np.abs(g - th[:, :p])) < 1e-12 and np.max(np.abs(b - th[:, p:])) < 1e-12
    assert np.max(np.abs(e - elast)) < 1e-12
    assert np.array_equal(st, np.where(done > 0, done - 1, steps))


def test_learned_curvature_pipeline_beats_plain():
    p, steps, lr = 4, 100, 0.05
    train = _graphs(768, [8, 10, 12], 3)
    held = _graphs(64, [10, 12], 4)
    g0, b0 = linear_ramp(p)
    qb = QaoaBatch(train, p, "f32")
    g, b, _, _ = qb.optimize(np.tile(g0, (len(train), 1)), np.tile(b0, (len(train), 1)), steps, lr)
    warm = WarmStart(p)
    warm.fit(train, g, b, chunks=4, chunk_steps=300)
    eig = warm.fit_curvature(train, g, b)
    assert all(np.all(w < 0) for w in eig.values())          # a maximum: negative curvature
    hb = QaoaBatch(held, p, "f32")
    G0, B0 = np.tile(g0, (len(held), 1)), np.tile(b0, (len(held), 1))
    _, _, target, _ = hb.optimize(G0, B0, steps, lr)
    _, _, e_ramp, st_ramp = hb.optimize(G0, B0, steps, lr, target=target, rtol=1e-5)
    pg, pb = warm.predict(held)
    _, _, e_wp, st_wp = hb.optimize_precond(pg, pb, warm.preconditioners(held), steps, 0.8, target=target, rtol=1e-5)
    assert np.mean(e_wp >= target * (1 - 1e-5)) >= 0.9
    assert np.median(st_wp) < 0.5 * np.median(st_ramp), (np.median(st_wp), np.median(st_ramp))


def test_convergence_rule_preconditioned_matches_host_loop():
    """run_qaoa's rule (qaoa.rs:266-269): an instance stops once its energy changed by less
    than tol in a step; the preconditioned device loop against the same loop on the host."""
    graphs = _graphs(5, [8, 10, 12], 8)
    p, steps, tol = 2, 12, 1e-3
    g0, b0 = linear_ramp(p)
    G, B = np.tile(g0, (5, 1)), np.tile(b0, (5, 1))
    r = np.random.default_rng(3)
    A = r.normal(size=(5, 2 * p, 2 * p))
    P = 0.01 * (np.einsum('kij,klj->kil', A, A) + np.eye(2 * p))
    qb = QaoaBatch(graphs, p, "f64")
    qb.set_convergence(tol)
    g, b, e, st = qb.optimize_precond(G, B, P, steps, 0.8)
    th = np.concatenate([G, B], axis=1)
    alpha = np.full(5, 0.8)
    eprev = np.full(5, -1e300)
    done = np.zeros(5, dtype=int)
    elast = np.zeros(5)
    for t in range(steps + 1):
        en, gr = qb.gradient(th[:, :p], th[:, p:])
        for k in range(5):
            if done[k]:
                continue
            elast[k] = en[k]
            if abs(en[k] - eprev[k]) < tol:
                done[k] = t + 1
                continue
            if t == steps:
                continue
            if en[k] < eprev[k]:
                alpha[k] *= 0.5
            eprev[k] = en[k]
            th[k] += alpha[k] * (P[k] @ gr[k])
    assert (st < steps).any()                      # the rule stopped someone early
    assert np.max(np.abs(g - th[:, :p])) < 1e-12 and np.max(np.abs(b - th[:, p:])) < 1e-12
    assert np.max(np.abs(e - elast)) < 1e-12
    assert np.array_equal(st, np.where(done > 0, done - 1, steps))


def test_convergence_rule_adam_stops_at_the_first_small_change():
    graphs = _graphs(6, [8, 10], 9)
    p, steps, lr = 2, 14, 0.05
    g0, b0 = linear_ramp(p)
    G, B = np.tile(g0, (6, 1)), np.tile(b0, (6, 1))
    qb = QaoaBatch(graphs, p, "f64")
    energy = np.stack([qb.optimize(G, B, s, lr)[2] for s in range(steps + 1)])   # energy after s updates
    # a tolerance that half of the steps' energy changes fall below, so some instances stop early
    tol = float(np.median(np.abs(np.diff(energy, axis=0))))
    qb.set_convergence(tol)
    _, _, e, st = qb.optimize(G, B, steps, lr)
    qb.set_convergence(0.0)
    for i in range(6):
        small = [s for s in range(1, steps + 1) if abs(energy[s, i] - energy[s - 1, i]) < tol]
        want = small[0] if small else steps
        assert st[i] == want, (i, st[i], want)
        assert abs(e[i] - energy[want, i]) < 1e-12
    assert (st < steps).any()
