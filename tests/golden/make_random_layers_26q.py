"""Generate tests/golden/random_layers_26q_seed1.npz: the oracle's 26-qubit random-layer state.

Circuit: the config-2 random-layer generator (ruqu_b200.workloads.random_layer_circuit) at
26 qubits, 20 layers, seed 1 -- Rz(theta) and Rx(phi) on every qubit per layer, then the
CNOT brickwork -- on the oracle's f64 engine (the restated reference kernels, state.rs:214-276,
gate by gate; the OpenMP variant of the same loops, which gives identical numbers, since
every amplitude is computed by the same expression in the same order), from |0...0>.
The full state (1 GiB) is too large to commit, so the fixture keeps:
  * amps      -- the amplitudes at 16384 indices drawn from the Philox stream (seed 26,
                 stream 6), with the indices;
  * z         -- <Z_q> for every qubit (state.rs:362-400 on the full state);
  * blocks    -- sum |a|^2 over each of the 256 consecutive blocks of 2^18 amplitudes;
  * sha256    -- of the full f64 amplitude vector's bytes (identifies this oracle output).
Run from the repository root (a few minutes on 8 cores):
    python tests/golden/make_random_layers_26q.py
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from ruqu_b200 import rng, workloads  # noqa: E402

N, LAYERS, SEED, SAMPLES = 26, 20, 1, 16384


def sample_indices():
    return np.unique((rng.Stream(26, 6).take(SAMPLES) * (1 << N)).astype(np.int64))


def main():
    gates = workloads.random_layer_circuit(N, LAYERS, SEED)
    st = oracle.OracleState(N, oracle.RQ_F64, 0)
    st.apply(gates, parallel=True)
    a = st.amplitudes()
    idx = sample_indices()
    p = a.real ** 2 + a.imag ** 2
    z = np.array([p[((np.arange(1 << N) >> q) & 1) == 0].sum() - p[((np.arange(1 << N) >> q) & 1) == 1].sum()
                  for q in range(N)])
    blocks = p.reshape(256, -1).sum(axis=1)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "random_layers_26q_seed1.npz")
    np.savez_compressed(out, indices=idx, amps=a[idx], z=z, blocks=blocks,
                        sha256=np.array(hashlib.sha256(a.tobytes()).hexdigest()),
                        meta=np.array([N, LAYERS, SEED]))
    print("max|a| %.3e  norm %.15f  gates %d" % (np.abs(a).max(), p.sum(), len(gates)))


if __name__ == "__main__":
    main()
