"""Batched QAOA-MaxCut engine vs the oracle (needs a GPU).

Energies are the oracle's evaluate_qaoa_cost restatement (qaoa.rs:179-201, per-edge
ZZ expectations of the gate-by-gate circuit); tolerance 1e-10 absolute for f64
states and 1e-5 x |E| for f32 states (FP64 accumulation of f32 amplitudes).
Best-cut shots are bit-exact against the oracle's sampler fed the same device
probability vector with the same seeds.
"""
import json
import math
import os

import numpy as np
import pytest

import oracle
from ruqu_b200 import rng, workloads
from ruqu_b200.batch import QaoaBatch

pytestmark = pytest.mark.gpu


def _graphs(sizes, seed):
    st = rng.Stream(seed, 2)
    out = []
    r = np.random.default_rng(seed)
    for n in sizes:
        if n % 2 == 0 and n >= 4:
            out.append((n, workloads.random_3regular_graph(n, st)))
        else:   # odd n: random simple graph with ~1.5 n edges
            pairs = [(i, j) for i in range(n) for j in range(i + 1, n)]
            pick = r.choice(len(pairs), size=min(len(pairs), (3 * n) // 2), replace=False)
            out.append((n, [pairs[k] for k in sorted(pick)]))
    return out


def _cut(bits, edges):
    return sum(1 for u, v in edges if ((bits >> u) ^ (bits >> v)) & 1)


def _best_from_oracle(probs, n, edges, seed, shots):
    bits = oracle.tree_sample(probs, n, list(range(n)), seed, shots)
    cuts = np.array([_cut(int(b), edges) for b in bits])
    k = int(np.argmax(cuts))          # first index of the maximum
    return int(bits[k]), int(cuts[k])


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("p", [1, 3])
def test_batch_energies_and_shots_match_oracle(prec, p):
    sizes = [6, 7, 8, 10, 12, 13, 14, 16] if prec == "f64" else [7, 8, 10, 12, 13, 14, 16]
    graphs = _graphs(sizes, 11 + p)
    nsets = 3
    r = np.random.default_rng(p)
    gam = r.uniform(0, math.pi, size=(len(graphs), nsets, p))
    bet = r.uniform(0, math.pi / 2, size=(len(graphs), nsets, p))
    qb = QaoaBatch(graphs, p, prec)
    shots, seed = 512, 1234
    out = qb.run(gam, bet, shots=shots, seed=seed)
    for k, (n, e) in enumerate(graphs):
        ew = [(u, v, 1.0) for u, v in e]
        for s in range(nsets):
            want = oracle.qaoa_cost(n, ew, gam[k, s], bet[k, s])
            tol = 1e-10 if prec == "f64" else 1e-5 * max(1, len(e))
            assert abs(out["energies"][k, s] - want) < tol, (n, s, out["energies"][k, s], want)
            assert out["best_cut"][k, s] == _cut(int(out["best_bits"][k, s]), e)
    # the largest size class runs last, so its circuits are still on the device:
    # their shots are bit-exact against the oracle sampler on the same probabilities
    k = len(graphs) - 1
    n, e = graphs[k]
    for s in range(nsets):
        c = k * nsets + s
        a = qb.state(c)
        probs = a.real * a.real + a.imag * a.imag
        assert _best_from_oracle(probs, n, e, seed + (c << 32), shots) == \
            (int(out["best_bits"][k, s]), int(out["best_cut"][k, s]))


def test_batch_waves_give_the_same_energies():
    graphs = _graphs([14, 14, 16, 16, 16], 5)
    r = np.random.default_rng(9)
    gam = r.uniform(0, math.pi, size=(len(graphs), 4))
    bet = r.uniform(0, math.pi / 2, size=(len(graphs), 4))
    a = QaoaBatch(graphs, 4, "f32")
    ea = a.run(gam, bet)["energies"]
    b = QaoaBatch(graphs, 4, "f32")
    b.set_state_budget(1 << 19)          # one 2^16-amplitude f32 state per wave
    eb = b.run(gam, bet)["energies"]
    assert np.max(np.abs(ea - eb)) == 0.0


def _golden():
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "qaoa_energies_n18_24.json")) as f:
        return json.load(f)


def test_batch_energies_n18_to_24_match_oracle_fixture():
    """The config's large sizes, where the engine streams states through HBM and splits
    the cost phase over register, thread and tile bits: three random 3-regular graphs for
    each n in {18, 20, 22, 24} at p = 4 (the seeded config generator, count 400, seed 17),
    in one batch with every other size class, against the oracle's f64 evaluate_qaoa_cost
    restatement (tests/golden/qaoa_energies_n18_24.json, made by make_qaoa_energies.py):
    f32 states within 1e-5 x |E|; one graph of n = 20 and one of n = 22 also on f64 states
    within 1e-10."""
    g = _golden()
    inst = workloads.qaoa_instances(g["count"], g["seed"])
    picked = [inst[e["index"]] for e in g["entries"]]
    for x, e in zip(picked, g["entries"]):
        assert x["n"] == e["n"] and len(x["edges"]) == e["edges"]
    graphs = [(x["n"], [(u, v) for u, v, _ in x["edges"]]) for x in picked]
    gam = np.array([x["gammas"] for x in picked])
    bet = np.array([x["betas"] for x in picked])
    out = QaoaBatch(graphs, 4, "f32").run(gam, bet)["energies"]
    for k, e in enumerate(g["entries"]):
        assert abs(out[k] - e["energy"]) < 1e-5 * e["edges"], (e["n"], out[k], e["energy"])
    sel = [next(k for k, e in enumerate(g["entries"]) if e["n"] == n) for n in (20, 22)]
    out64 = QaoaBatch([graphs[k] for k in sel], 4, "f64").run(gam[sel], bet[sel])["energies"]
    for j, k in enumerate(sel):
        assert abs(out64[j] - g["entries"][k]["energy"]) < 1e-10


def test_batch_best_cut_of_every_wave_matches_oracle_sampler():
    """Random 3-regular graphs with n uniform over {12..18}, p = 4, 1024 shots, run with a
    state budget that forces several waves; every circuit's best cut (bits and value) must
    equal the oracle's tree sampler on that circuit's probabilities.  The probabilities come
    from a batch of that one graph, whose state stays on the device (a circuit's amplitudes do
    not depend on the batch it runs in -- the energies of the two runs are bit-identical -- and
    its shot seed depends only on its index)."""
    inst = workloads.qaoa_instances(24, 3, n_values=(12, 14, 16, 18))
    graphs = [(x["n"], [(u, v) for u, v, _ in x["edges"]]) for x in inst]
    gam = np.array([x["gammas"] for x in inst])
    bet = np.array([x["betas"] for x in inst])
    waved = QaoaBatch(graphs, 4, "f32")
    waved.set_state_budget(1 << 22)            # 4 MB: two 2^18 f32 states per wave
    out = waved.run(gam, bet, shots=1024, seed=7)
    whole = QaoaBatch(graphs, 4, "f32")
    ref = whole.run(gam, bet, shots=1024, seed=7)
    assert np.array_equal(out["energies"], ref["energies"])
    for k, (n, e) in enumerate(graphs):
        assert 0.0 <= out["energies"][k] <= len(e)
        assert out["best_cut"][k] == _cut(int(out["best_bits"][k]), e)
        one = QaoaBatch([graphs[k]], 4, "f32")
        assert one.run(gam[k:k + 1], bet[k:k + 1])["energies"][0] == out["energies"][k]
        a = one.state(0)
        probs = a.real * a.real + a.imag * a.imag
        assert _best_from_oracle(probs, n, e, 7 + (k << 32), 1024) == (int(out["best_bits"][k]),
                                                                         int(out["best_cut"][k])), (k, n)


def test_repeated_runs_replay_one_graph_with_identical_results():
    """rq_qaoa_batch_run / _gradient as CUDA graphs: the first run of a shape is plain, the
    second captures and launches the graph, later ones replay it; energies, shots and
    gradients equal those of a batch that never uses graphs, for new angles every run, and
    a new shape (other shot count) runs plainly again."""
    graphs = _graphs([10, 12, 12, 14, 16], 21)
    r = np.random.default_rng(4)
    a = QaoaBatch(graphs, 3, "f32")
    plain = QaoaBatch(graphs, 3, "f32")
    plain.set_graphs(False)
    flags = []
    for it in range(4):
        gam = r.uniform(0, math.pi, size=(len(graphs), 2, 3))
        bet = r.uniform(0, math.pi / 2, size=(len(graphs), 2, 3))
        x = a.run(gam, bet, shots=256, seed=77)
        flags.append(a.last_graph()["replayed"])
        y = plain.run(gam, bet, shots=256, seed=77)
        assert not plain.last_graph()["replayed"]
        for k in ("energies", "best_bits", "best_cut"):
            assert np.array_equal(x[k], y[k]), (it, k)
    assert flags == [False, True, True, True]
    assert a.last_graph()["kernels"] > 5
    x = a.run(gam, bet, shots=128, seed=77)
    assert not a.last_graph()["replayed"]
    assert np.array_equal(x["energies"], plain.run(gam, bet, shots=128, seed=77)["energies"])
    for it in range(3):
        g1 = r.uniform(0, math.pi, size=(len(graphs), 3))
        b1 = r.uniform(0, math.pi / 2, size=(len(graphs), 3))
        ea, ga = a.gradient(g1, b1)
        eb, gb = plain.gradient(g1, b1)
        assert np.array_equal(ea, eb) and np.array_equal(ga, gb)
        assert a.last_graph()["replayed"] == (it > 0)
