"""ruqu-wasm's qaoa_maxcut by semantics on the device (needs a GPU): probabilities and
the expected cut against the oracle's QAOA restatement (qaoa.rs:125-201), f64 states,
1e-12 (probabilities) and 1e-10 (expected cut)."""
import numpy as np
import pytest

import oracle
from ruqu_b200 import rng, workloads
from ruqu_b200.qaoa import qaoa_maxcut

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,p,seed", [(4, 1, 1), (8, 2, 2), (12, 3, 3)])
def test_matches_the_oracle(n, p, seed):
    edges = workloads.random_3regular_graph(n, rng.Stream(seed, 2))
    flat = [int(x) for e in edges for x in e]
    r = np.random.default_rng(seed)
    gammas, betas = r.uniform(0, np.pi, p), r.uniform(0, np.pi / 2, p)
    out = qaoa_maxcut(n, flat, p, gammas, betas, seed=7)
    we = [(u, v, 1.0) for u, v in edges]
    assert np.max(np.abs(out["probabilities"] - oracle.qaoa_probabilities(n, we, gammas, betas))) < 1e-12
    assert abs(out["expected_cut"] - oracle.qaoa_cost(n, we, gammas, betas)) < 1e-10


def test_no_edges():
    out = qaoa_maxcut(3, [], 1, [0.4], [0.2])
    assert out["expected_cut"] == 0.0
    assert abs(out["probabilities"].sum() - 1.0) < 1e-12
