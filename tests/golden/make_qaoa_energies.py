"""Generate tests/golden/qaoa_energies_n18_24.json: oracle energies of batched-QAOA instances.

The instances are the seeded config-3 generator's (ruqu_b200.workloads.qaoa_instances,
count 400, seed 17: random 3-regular graphs, unit weights, p = 4, gamma ~ U[0, pi),
beta ~ U[0, pi/2)); the first three of each size n in {18, 20, 22, 24} are kept.  Each
energy is the oracle's restatement of evaluate_qaoa_cost (qaoa.rs:179-201: the
gate-by-gate f64 circuit of build_qaoa_circuit, then the per-edge ZZ expectations), which
takes seconds per graph at these sizes -- too slow to rerun inside the GPU tests, hence
the fixture.  Run from the repository root: python tests/golden/make_qaoa_energies.py
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from ruqu_b200 import workloads  # noqa: E402

COUNT, SEED, PER_SIZE = 400, 17, 3


def main():
    inst = workloads.qaoa_instances(COUNT, SEED)
    entries = []
    for n in (18, 20, 22, 24):
        idx = [k for k, x in enumerate(inst) if x["n"] == n][:PER_SIZE]
        for k in idx:
            x = inst[k]
            e = oracle.qaoa_cost(n, x["edges"], x["gammas"], x["betas"])
            entries.append({"index": k, "n": n, "edges": len(x["edges"]), "energy": e})
            print(n, k, e, flush=True)
    out = {"generator": "ruqu_b200.workloads.qaoa_instances", "count": COUNT, "seed": SEED, "p": 4,
           "oracle": "evaluate_qaoa_cost restatement, f64", "entries": entries}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "qaoa_energies_n18_24.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
