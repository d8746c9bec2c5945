"""Benchmark of the state-vector hot path: 30-qubit random-layer circuit, HBM GB/s.

Workload: random-layer circuit on 30 qubits (2^30 amplitudes, complex f32 =
8 GiB), 20 layers, seed 1; each layer is Rz(theta)+Rx(phi) on every qubit
and a CNOT brickwork (even pairs on even layers, odd pairs on odd layers).
A step is one full simulation: |0...0> initialisation plus the 20 layers.

value   -- per-gate-layer HBM GB/s: (S for the |0> write + 2S per layer, the
           read and write of the state that one pass per layer needs) / device
           time of the step (CUDA events on the state's stream), with the
           prepared plan resident on the GPU; summed over ranks / max time.
e2e     -- the same bytes through the public API with host buffers: reset,
           apply(host gate list), read <Z_i> for all qubits back to the host;
           wall-clock per step.
roofline-- the dominant kernel (the sweep kernel the plan launches): 2S per
           launch / its average launch time, against the measured HBM copy
           bandwidth.
variants-- one run of each execution mode (unfused per-gate kernels, CUDA-core
           sweeps, 3xTF32 and one-pass TF32 tensor-core sweeps) with its
           per-layer GB/s and its max-abs amplitude error against the complex
           f64 run of the same circuit.

N>1 ranks (torchrun) run independent replicas (the state does not shard on
one node at this size): weak scaling, no collective on the data path.
`--impl reference` times the CPU restatement of the reference's kernels on
all host cores (bounded sample of the same circuit) on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "30q HBM GB/s"
UNIT = "GB/s"
FALLBACK_HBM_GBS = 6650.0


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--layers", type=int, default=20)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--precision", choices=["f32", "f64"], default="f32")
    ap.add_argument("--mode", choices=["auto", "per_gate", "sweep", "tc", "tc_fast", "tc16"], default="auto")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-qaoa", action="store_true", help="skip the batched QAOA leg")
    ap.add_argument("--qaoa-instances", type=int, default=2048)
    ap.add_argument("--qaoa-sizes", default="12,14,16,18,20,22,24",
                    help="graph sizes of the batched QAOA leg (the config's n uniform over {12..24})")
    ap.add_argument("--no-vqe", action="store_true", help="skip the batched VQE leg")
    ap.add_argument("--vqe-sets", type=int, default=512)
    ap.add_argument("--no-warm", action="store_true", help="skip the warm-start leg")
    ap.add_argument("--no-variants", action="store_true", help="skip the per-mode runs and the f64 comparison")
    ap.add_argument("--no-sampling", action="store_true", help="skip the <Z_i> + shots leg on the final state")
    ap.add_argument("--no-small", action="store_true", help="skip the 20-qubit f64 circuit leg")
    ap.add_argument("--warm-train", type=int, default=2048, help="training graphs for the warm start")
    ap.add_argument("--warm-train-sizes", default="12,14,16,18,20,22",
                    help="graph sizes of the warm start's training graphs")
    ap.add_argument("--warm-eval", type=int, default=96, help="held-out graphs for the warm start")
    ap.add_argument("--warm-eval-sizes", default="16,18,20,22,24,26",
                    help="graph sizes of the held-out graphs (the config's n in {16..26})")
    ap.add_argument("--warm-extra", action="store_true",
                    help="also run the 50-step-budget and run_qaoa-convergence-rule arms")
    return ap.parse_args()


def _peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def _workload_desc(a):
    return (f"random-layer circuit, {a.qubits} qubits, {a.layers} layers, seed {a.seed}, "
            f"complex {a.precision} state (Rz+Rx on every qubit, CNOT brickwork)")


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.proc = None
        self.path = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 7:
                continue
            try:
                sm.append(float(p[0]))
                mx = float(p[1])
            except ValueError:
                continue
            for name, v in zip(names, p[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    from ruqu_b200.dist import world
    return world()


def _gate_kinds(gates):
    """(one-qubit gates, two-qubit gates) of a gate list."""
    one = [g for g in gates if g[0] != 12]
    two = [g for g in gates if g[0] == 12]
    return one, two


def cpu_circuit_time(a, parallel: bool, n_one: int, n_two: int, st=None, start: int = 0):
    """Time n_one one-qubit gates and n_two CNOTs of the benchmark circuit on the oracle
    (the restated reference kernels, one pass over the state per gate), each gate timed on
    its own, and extrapolate to the whole circuit: circuit seconds = (#1q gates) x mean 1q
    time + (#CNOTs) x mean CNOT time.  Returns (circuit seconds, timed seconds, cores, the
    state, per-kind mean seconds)."""
    import oracle
    from ruqu_b200 import workloads
    gates = workloads.random_layer_circuit(a.qubits, a.layers, a.seed)
    one, two = _gate_kinds(gates)
    if st is None:
        prec = oracle.RQ_F32 if a.precision == "f32" else oracle.RQ_F64
        st = oracle.OracleState(a.qubits, prec, 0)
    t_one, t_two = [], []
    for k in range(n_one):
        g = one[(start * n_one + k) % len(one)]
        t0 = time.perf_counter()
        st.apply([g], parallel=parallel)
        t_one.append(time.perf_counter() - t0)
    for k in range(n_two):
        g = two[(start * n_two + k) % len(two)]
        t0 = time.perf_counter()
        st.apply([g], parallel=parallel)
        t_two.append(time.perf_counter() - t0)
    m1 = sum(t_one) / max(1, len(t_one))
    m2 = sum(t_two) / max(1, len(t_two))
    circuit_s = len(one) * m1 + len(two) * m2
    cores = oracle.num_threads() if parallel else 1
    return circuit_s, sum(t_one) + sum(t_two), cores, st, (m1, m2)


def cpu_baseline_sample(a, parallel: bool):
    """The CPU baseline of the GPU arm: the oracle's scalar reference kernels (1 thread) on
    two one-qubit gates and one CNOT of the benchmark circuit, extrapolated to the whole
    circuit; reported in the GPU arm's own unit (per-layer bytes / circuit time).
    Returns (GB/s, circuit seconds, timed seconds, cores, sample description)."""
    S = (1 << a.qubits) * (8 if a.precision == "f32" else 16)
    layer_bytes = S + 2 * S * a.layers
    circuit_s, timed_s, cores, _, (m1, m2) = cpu_circuit_time(a, parallel, 2, 1)
    desc = (f"2 one-qubit gates and 1 CNOT of the {a.qubits}-qubit circuit on a {a.precision} state, each one "
            f"pass of the {'OpenMP restatement of the reference parallel kernels' if parallel else 'scalar reference kernels'}"
            f" ({cores} thread(s)); mean {m1 * 1e3:.0f} ms per 1q gate, {m2 * 1e3:.0f} ms per CNOT; circuit time "
            f"extrapolated by gate counts; value = (S + 2S x layers) / circuit time, the GPU arm's byte count")
    return layer_bytes / circuit_s / 1e9, circuit_s, timed_s, cores, desc


def qaoa_batch_leg(a, ws, rank, with_cpu):
    """Batched QAOA-MaxCut: 2048 random 3-regular graphs, n uniform over {12,...,24},
    unit weights, p = 4, gamma ~ U[0,pi), beta ~ U[0,pi/2) (seed 2), complex f32
    states, <C> in FP64, 1024 shots per graph -> best-cut bitstring.  Instances
    are sharded over ranks (rank r takes r, r+N, ...)."""
    import numpy as np

    from ruqu_b200 import workloads
    from ruqu_b200.batch import QaoaBatch
    from ruqu_b200.dist import shard
    sizes = tuple(int(x) for x in a.qaoa_sizes.split(","))
    inst = workloads.qaoa_instances(a.qaoa_instances, 2, n_values=sizes)
    mine = shard(inst, rank, ws)
    graphs = [(x["n"], [(u, v) for u, v, _ in x["edges"]]) for x in mine]
    gam = np.array([x["gammas"] for x in mine])
    bet = np.array([x["betas"] for x in mine])
    qb = QaoaBatch(graphs, 4, "f32")
    qb.run(gam, bet, shots=1024, seed=11)            # warm-up (allocation, first launches)
    ms, wall, profs = [], [], []
    for _ in range(3):
        t0 = time.perf_counter()
        out = qb.run(gam, bet, shots=1024, seed=11)
        wall.append(time.perf_counter() - t0)
        ms.append(qb.last_ms())
        profs.append(qb.last_profile())
    dev_ms = min(ms)
    prof = profs[int(np.argmin(ms))]
    peak, peak_kind = _peak()
    sweep_gbs = prof["sweep_bytes"] / (prof["sweep_ms"] / 1e3) / 1e9
    sample_gbs = prof["sample_bytes"] / (prof["sample_ms"] / 1e3) / 1e9
    res = {"workload": "batched QAOA-MaxCut, %d random 3-regular graphs, n in {%s}, p=4, f32 states, "
                       "1024 shots each, best cut" % (a.qaoa_instances, a.qaoa_sizes),
           "circuits_per_rank": len(mine), "device_ms": dev_ms, "wall_ms": 1e3 * min(wall),
           "evals_per_s": len(mine) * ws / (dev_ms / 1e3),
           "evals_per_s_e2e": len(mine) * ws / min(wall),
           "mean_energy": float(np.mean(out["energies"])), "mean_best_cut": float(np.mean(out["best_cut"])),
           "roofline": {"bound": "hbm", "kernel": "k_batch_sweep (all size classes and waves)",
                        "achieved": sweep_gbs, "peak": peak, "unit": "GB/s", "frac": sweep_gbs / peak,
                        "peak_kind": peak_kind, "bytes": prof["sweep_bytes"], "kernel_ms": prof["sweep_ms"],
                        "bytes_definition": "per circuit and sweep: S written by the initialising sweep, 2S "
                                            "(read + write) for every other sweep; S = 2^n x 8 B"},
           "sampling": {"kernels": "k_leaf_fold / k_fold / k_sample (1024 shots per circuit)",
                        "achieved_gbs": sample_gbs, "bytes": prof["sample_bytes"], "kernel_ms": prof["sample_ms"],
                        "frac": sample_gbs / peak},
           "device_ms_outside_kernels": dev_ms - prof["sweep_ms"] - prof["sample_ms"]}
    # exact gradients of the same circuits: forward sweeps, then k_batch_adjoint over psi and lambda
    qb.gradient(gam, bet)
    gms, gprofs = [], []
    for _ in range(3):
        qb.gradient(gam, bet)
        gms.append(qb.last_ms())
        gprofs.append(qb.last_profile())
    gp = gprofs[int(np.argmin(gms))]
    res["adjoint_gradient"] = {
        "device_ms": min(gms), "gradients_per_s": len(mine) * ws / (min(gms) / 1e3),
        "roofline": {"bound": "hbm", "kernel": "k_batch_adjoint (psi and lambda through the reversed program)",
                     "achieved": gp["adjoint_bytes"] / (gp["adjoint_ms"] / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": gp["adjoint_bytes"] / (gp["adjoint_ms"] / 1e3) / 1e9 / peak, "peak_kind": peak_kind,
                     "bytes": gp["adjoint_bytes"], "kernel_ms": gp["adjoint_ms"],
                     "bytes_definition": "per circuit and backward sweep: read + write of psi and lambda (4S), "
                                         "3S for the sweep that builds lambda = C psi instead of loading it"}}
    if with_cpu:
        import oracle
        t_by_n = {}
        present = sorted({x["n"] for x in inst})
        timed = [n for n in present if n <= 18] or present[:1]
        for n in timed:
            x = next(y for y in inst if y["n"] == n)
            t0 = time.perf_counter()
            oracle.qaoa_cost(n, x["edges"], x["gammas"], x["betas"])
            t_by_n[n] = time.perf_counter() - t0
        for n in present:   # each +2 qubits: 4x the amplitudes, (n+2)/n the gates
            if n not in t_by_n:
                m = max(k for k in t_by_n if k < n)
                t = t_by_n[m]
                for k in range(m, n, 2):
                    t *= 4.0 * (k + 2) / k
                t_by_n[n] = t
        total = sum(t_by_n[x["n"]] for x in inst)
        res["cpu_baseline"] = {"value": len(inst) / total, "unit": "QAOA evals/s", "cores": 1, "kind": "port",
                               "sample": "one evaluate_qaoa_cost (reference f64 engine, energy only, no shots) "
                                         "per n in {%s} timed; larger n scaled by 4(n+2)/n per +2 qubits; summed "
                                         "over the %d instances" % (",".join(map(str, timed)), len(inst))}
    return res


def vqe_batch_leg(a, ws, rank, with_cpu):
    """Batched VQE energies + parameter-shift gradients: 16 qubits, H = 200 random
    Pauli strings (seed 3), depth-8 Ry + CZ-ladder ansatz (128 parameters), 512
    parameter sets ~ U[-pi, pi) (seed 4), each with 256 shifted evaluations:
    131,584 circuits, f32 states, energies in FP64.  Sets are sharded over ranks."""
    import numpy as np

    from ruqu_b200 import workloads
    from ruqu_b200.batch import VqeBatch
    n, depth = 16, 8
    coeffs, strings = workloads.pauli_hamiltonian(n, 200, 3)
    from ruqu_b200.dist import shard
    params = shard(workloads.vqe_parameter_sets(a.vqe_sets, n * depth, 4), rank, ws)
    vb = VqeBatch(n, depth, coeffs, strings, "f32")
    vb.run(params[:2], gradient=True)           # warm-up
    ms, wall, profs = [], [], []
    for _ in range(2):
        t0 = time.perf_counter()
        e, g = vb.run(params, gradient=True)
        wall.append(time.perf_counter() - t0)
        ms.append(vb.last_ms())
        profs.append(vb.last_profile())
    prof = profs[int(np.argmin(ms))]
    circuits = len(params) * (1 + 2 * n * depth)
    # the same energies and gradients by the adjoint pass (one forward, lambda = H psi, one backward)
    vb.run(params[:2], gradient="adjoint")
    ams, aprofs = [], []
    for _ in range(3):
        ea, ga = vb.run(params, gradient="adjoint")
        ams.append(vb.last_ms())
        aprofs.append(vb.last_profile())
    aprof = aprofs[int(np.argmin(ams))]
    peak, peak_kind = _peak()
    scale = float(np.sum(np.abs(coeffs)))
    res = {"workload": "batched VQE, 16 qubits, 200-term Pauli Hamiltonian, depth-8 Ry+CZ ansatz, %d parameter "
                       "sets x 257 parameter-shift circuits, f32 states" % a.vqe_sets,
           "circuits_per_rank": circuits, "device_ms": min(ms), "wall_ms": 1e3 * min(wall),
           "circuits_per_s": circuits * ws / (min(ms) / 1e3), "mean_energy": float(np.mean(e)),
           "gradient_sets_per_s_shift": len(params) * ws / (min(ms) / 1e3),
           "roofline": {"bound": "hbm", "kernel": "k_batch_sweep (ansatz evolution of all 131,584 circuits)",
                        "achieved": prof["sweep_bytes"] / (prof["sweep_ms"] / 1e3) / 1e9, "peak": peak,
                        "unit": "GB/s",
                        "frac": prof["sweep_bytes"] / (prof["sweep_ms"] / 1e3) / 1e9 / peak,
                        "peak_kind": peak_kind, "bytes": prof["sweep_bytes"], "kernel_ms": prof["sweep_ms"],
                        "note": "waves of ~96 MB of states are sized to stay in L2, so these bytes are mostly "
                                "L2 traffic: a fraction above 1 of the HBM copy peak is possible and expected"},
           "energy_pass": {"kernel": "k_vqe_energy_tiles", "flops": prof["energy_flops"],
                           "kernel_ms": prof["energy_ms"],
                           "achieved_tflops": prof["energy_flops"] / (prof["energy_ms"] / 1e3) / 1e12,
                           "flops_definition": "8 per Pauli string and amplitude: one complex product "
                                               "conj(a[i^x]) a[i] and its FP64 accumulation (CUDA cores, FP32 "
                                               "products, FP64 sums; no measured peak for this mix)"},
           "adjoint": {"device_ms": min(ams), "gradient_sets_per_s": len(params) * ws / (min(ams) / 1e3),
                       "kernel_ms": aprof["adjoint_ms"], "bytes": aprof["adjoint_bytes"],
                       "achieved_gbs": aprof["adjoint_bytes"] / max(1e-9, aprof["adjoint_ms"] / 1e3) / 1e9,
                       "speedup_vs_shift": min(ms) / min(ams),
                       "max_abs_grad_diff_vs_shift_rel": float(np.max(np.abs(ga - g))) / scale,
                       "energies_identical": bool(np.array_equal(ea, e))}}
    if with_cpu:
        import oracle
        t0 = time.perf_counter()
        k = 2
        for s in range(k):
            oracle.circuit_energy(n, workloads.hea_ry_cz(n, depth, params[s]), coeffs, strings)
        dt = (time.perf_counter() - t0) / k
        res["cpu_baseline"] = {"value": 1.0 / dt, "unit": "circuits/s", "cores": 1, "kind": "port",
                               "sample": "evaluate_energy of 2 ansatz circuits on the reference f64 engine "
                                         "(gate by gate, one pass per Pauli term), averaged"}
    return res


def warmstart_leg(a, ws, rank, with_cpu=False):
    """Learned warm start vs linear ramp for QAOA p = 4.  The config asks for 200k training
    pairs and 4096 held-out graphs with n in {16..26}; that many optimizer runs take tens of
    GPU-minutes (about 3 ms per Adam step of one 26-node graph), so the default leg keeps the
    sizes and scales the counts down (--warm-train / --warm-eval set them).
    Training: a.warm_train random 3-regular graphs with n in --warm-train-sizes, angles from
    the plain batched optimizer (linear ramp + 100 Adam steps, lr 0.05, exact adjoint
    gradients); the MLP (325 -> 256 -> 256 -> 8, BF16 tensor cores) learns the per-graph
    correction to the size trend of the optimal angles.
    Evaluation on a.warm_eval held-out graphs, n uniform over --warm-eval-sizes: the target of
    each graph is the energy of 200 plain Adam steps from the ramp; each arm then runs until
    every graph is within 1e-5 relative of its target (at most 200 steps; finished graphs
    leave the launches):
      plain            linear ramp + Adam (lr 0.05)
      warm + Adam      the MLP's angles + Adam (lr 0.005)
      learned pipeline the MLP's angles + ascent steps preconditioned by the learned curvature
                       (-H^-1 of the graph size's average Hessian at the training optima,
                       damping 0.8, halved on a fall)
      mean + curvature the size trend alone (no network) + the same preconditioned steps:
                       what the network itself adds is learned pipeline vs this arm
      ramp + curvature the linear ramp + the same preconditioned steps
    (--warm-extra adds the learned pipeline with a 50-step budget and both pipelines with
    run_qaoa's convergence rule).  solves/s = graphs that reached the target / device time of
    the arm (plus the MLP inference for the MLP arms).  The headline speedup is the learned
    pipeline against plain."""
    import numpy as np

    from ruqu_b200 import rng, workloads
    from ruqu_b200.batch import QaoaBatch
    from ruqu_b200.warmstart import WarmStart, linear_ramp
    p, lr, lr_warm = 4, 0.05, 0.005
    train_sizes = tuple(int(x) for x in a.warm_train_sizes.split(","))
    eval_sizes = tuple(int(x) for x in a.warm_eval_sizes.split(","))

    def graphs(count, sizes, seed):
        st = rng.Stream(seed, 2)
        sel = rng.Stream(seed, 3)
        return [(n, workloads.random_3regular_graph(n, st)) for n in
                (sizes[sel.randint(len(sizes))] for _ in range(count))]

    def reached(e, target):
        return e >= target * (1 - 1e-5)

    g0, b0 = linear_ramp(p)
    t0 = time.perf_counter()
    train = graphs(a.warm_train, train_sizes, 21)
    qb = QaoaBatch(train, p, "f32")
    g, b, _, _ = qb.optimize(np.tile(g0, (len(train), 1)), np.tile(b0, (len(train), 1)), 100, lr)
    gen_ms = qb.last_ms()
    warm = WarmStart(p)
    hist = warm.fit(train, g, b)
    warm.fit_curvature(train, g, b)
    from ruqu_b200.dist import shard
    held = shard(graphs(a.warm_eval, eval_sizes, 22), rank, ws)
    hb = QaoaBatch(held, p, "f32")
    G0, B0 = np.tile(g0, (len(held), 1)), np.tile(b0, (len(held), 1))
    opt_g, opt_b, target, _ = hb.optimize(G0, B0, 200, lr)
    setup_s = time.perf_counter() - t0
    arms = {}

    def arm(name, ms, e, steps):
        ok = reached(e, target)
        arms[name] = {"ms": ms, "reached": float(ok.mean()), "solves_per_s": float(ok.sum()) * ws / (ms / 1e3),
                      "median_steps": float(np.median(steps)), "max_steps": int(np.max(steps))}

    _, _, e, st = hb.optimize(G0, B0, 200, lr, target=target, rtol=1e-5)
    arm("plain", hb.last_ms(), e, st)
    warm.predict(held)                       # warm-up (host threads, device buffers)
    t1 = time.perf_counter()
    pg, pb = warm.predict(held)
    infer_ms = (time.perf_counter() - t1) * 1e3
    _, _, e, st = hb.optimize(pg, pb, 200, lr_warm, target=target, rtol=1e-5)
    arm("warm_adam", hb.last_ms() + infer_ms, e, st)
    P = warm.preconditioners(held)
    _, _, e, st = hb.optimize_precond(pg, pb, P, 200, 0.8, target=target, rtol=1e-5)
    arm("learned_pipeline", hb.last_ms() + infer_ms, e, st)
    mg, mb = warm.mean_angles(held)
    _, _, e, st = hb.optimize_precond(mg, mb, P, 200, 0.8, target=target, rtol=1e-5)
    arm("mean_curvature", hb.last_ms(), e, st)
    _, _, e, st = hb.optimize_precond(G0, B0, P, 200, 0.8, target=target, rtol=1e-5)
    arm("ramp_curvature", hb.last_ms(), e, st)
    if a.warm_extra:
        _, _, e, st = hb.optimize_precond(pg, pb, P, 50, 0.8, target=target, rtol=1e-5)
        arm("learned_pipeline_50_steps", hb.last_ms() + infer_ms, e, st)
        hb.set_convergence(1e-6)   # run_qaoa's rule (qaoa.rs:266-269): |dE| < 1e-6 stops an instance
        _, _, e, st = hb.optimize(G0, B0, 200, lr, target=target, rtol=1e-5)
        arm("plain_convergence_rule", hb.last_ms(), e, st)
        _, _, e, st = hb.optimize_precond(pg, pb, P, 200, 0.8, target=target, rtol=1e-5)
        arm("learned_pipeline_convergence_rule", hb.last_ms() + infer_ms, e, st)
        hb.set_convergence(0.0)
        # the network on label-free cycle statistics instead of the padded adjacency
        wc = WarmStart(p, encoding="cycles")
        hist_c = wc.fit(train, g, b)
        wc.precond = warm.precond
        t2 = time.perf_counter()
        cg, cb = wc.predict(held)
        infer_c = (time.perf_counter() - t2) * 1e3
        _, _, e, st = hb.optimize_precond(cg, cb, P, 200, 0.8, target=target, rtol=1e-5)
        arm("cycles_pipeline", hb.last_ms() + infer_c, e, st)
        # the same start with a safeguard: instances not at their target after K steps start
        # again from the size trend (the remaining budget, on a batch of those instances only)
        K = 12
        g1, b1, e1, st1 = hb.optimize_precond(cg, cb, P, K, 0.8, target=target, rtol=1e-5)
        ms = hb.last_ms() + infer_c
        left = np.flatnonzero(~reached(e1, target))
        e_all, st_all = e1.copy(), st1.astype(np.int64)
        if len(left):
            sb = QaoaBatch([held[i] for i in left], p, "f32")
            _, _, e2, st2 = sb.optimize_precond(mg[left], mb[left], P[left], 200 - K, 0.8, target=target[left],
                                                rtol=1e-5)
            ms += sb.last_ms()
            e_all[left] = e2
            st_all[left] = K + st2
        arm("cycles_then_trend", ms, e_all, st_all)
        arms["cycles_then_trend"]["restarted"] = int(len(left))
        arms["cycles_pipeline"]["mlp_val_error_vs_trend"] = min(hist_c) if hist_c else None
        arms["cycles_pipeline"]["median_start_distance"] = float(np.median(np.linalg.norm(
            np.concatenate([cg, cb], axis=1) - np.concatenate([opt_g, opt_b], axis=1), axis=1)))
    # start-point quality: distance of each start from the graph's own optimum (the plain run's)
    ng = np.array([n for n, _ in held])
    opt = np.concatenate([opt_g, opt_b], axis=1)
    dist = {"mlp": np.linalg.norm(np.concatenate([pg, pb], axis=1) - opt, axis=1),
            "mean": np.linalg.norm(np.concatenate([mg, mb], axis=1) - opt, axis=1)}
    by_size = {int(n): {"held_out": int((ng == n).sum()),
                        "median_start_distance_mlp": float(np.median(dist["mlp"][ng == n])),
                        "median_start_distance_mean": float(np.median(dist["mean"][ng == n]))}
               for n in sorted(set(ng.tolist()))}
    res = {"workload": "QAOA p=4 warm start vs linear ramp: train %d graphs n in {%s}, evaluate %d held-out graphs "
                       "n in {%s}; each arm runs until every graph is within 1e-5 of its 200-step plain Adam energy; "
                       "f32 states" % (a.warm_train, a.warm_train_sizes, a.warm_eval, a.warm_eval_sizes),
           "counts_note": "the config's 200k training pairs / 4096 held-out graphs are scaled down to keep the "
                          "default bench within minutes; sizes are the config's",
           "train_data_device_ms": gen_ms, "setup_s": setup_s, "warm_inference_ms": infer_ms,
           "mlp_val_error_vs_trend": min(hist) if hist else None,
           "mlp_val_error_definition": "held-out mean squared error of the network's correction, as a fraction "
                                       "of the residual variance around the size trend (below 1: the network "
                                       "predicts part of the per-graph correction)",
           "arms": arms, "by_size": by_size,
           "speedup": arms["learned_pipeline"]["solves_per_s"] / max(1e-9, arms["plain"]["solves_per_s"]),
           "speedup_network_vs_mean": arms["learned_pipeline"]["solves_per_s"] /
                                      max(1e-9, arms["mean_curvature"]["solves_per_s"]),
           "speedup_definition": "learned pipeline (MLP start + learned-curvature steps) vs plain (linear ramp + "
                                 "Adam), solves/s; speedup_network_vs_mean = learned pipeline vs the size trend "
                                 "with the same steps"}
    if with_cpu:
        # the plain method on the CPU restatement: Adam steps with central-difference gradients
        # of the oracle's evaluate_qaoa_cost (16 evaluations per step) on one 16-node graph,
        # 2 steps timed, scaled by the plain GPU arm's median step count
        import oracle
        n16 = next(x for x in held if x[0] == min(eval_sizes))
        edges = [(u, v, 1.0) for u, v in n16[1]]
        th = np.concatenate([g0, b0])
        t2 = time.perf_counter()
        for _ in range(2):
            for j in range(2 * p):
                for d in (1e-5, -1e-5):
                    tt = th.copy()
                    tt[j] += d
                    oracle.qaoa_cost(n16[0], edges, tt[:p], tt[p:])
        step_s = (time.perf_counter() - t2) / 2
        res["cpu_baseline"] = {"value": 1.0 / (step_s * arms["plain"]["median_steps"]), "unit": "solves/s",
                               "cores": 1, "kind": "port",
                               "sample": "2 Adam steps (16 oracle evaluate_qaoa_cost calls each, f64, n=%d) timed, "
                                         "scaled by the plain GPU arm's median steps (%g)"
                                         % (n16[0], arms["plain"]["median_steps"])}
    return res


# DRAM bytes (read + write) of one sweep launch measured by ncu on the 26-qubit
# case of this circuit, per tile; a launch moves every tile once, so the figure
# scales with the tile count (x16 from 26 to 30 qubits).
_NCU_BYTES_PER_TILE = {"k_sweep_tc": (537.133824e6 + 487.704576e6) / 2 ** 13,
                       "k_sweep": (537.2e6 + 485.1e6) / 2 ** 13,
                       "k_sweep_tc16": (537.199360e6 + 484.082176e6) / 2 ** 13}


_EXECUTED_AS = {1: "unfused per-gate kernels", 2: "CUDA-core sweeps", 3: "tensor-core sweeps (3xTF32)",
                4: "tensor-core sweeps (one TF32 pass)", 5: "tensor-core sweeps (3xFP16 split)"}
_KERNEL_OF = {2: "k_sweep (multi-gate sweep)", 3: "k_sweep_tc (tensor-core sweep, 3xTF32)",
              4: "k_sweep_tc (tensor-core sweep, one TF32 pass)", 5: "k_sweep_tc16 (tensor-core sweep, 3xFP16)"}


def _traffic_per_launch(a, stats):
    kern = {2: "k_sweep", 3: "k_sweep_tc", 4: "k_sweep_tc", 5: "k_sweep_tc16"}.get(stats["exec_mode"])
    if a.precision != "f32" or kern not in _NCU_BYTES_PER_TILE or stats["local_qubits"] != 13:
        return None
    return _NCU_BYTES_PER_TILE[kern] * 2 ** (a.qubits - 13)


def small_circuit_leg(with_cpu):
    """The reference's small configuration: 20 qubits, complex f64, 40 random layers
    (seed 0), then <Z_i> for every qubit and 4096 shots (a full simulator run with its
    read-out).  Device time through the public API (state created, gates applied from the
    host list, results back on the host), gates/s, per-layer GB/s; beside it the oracle's
    scalar f64 reference kernels on the same circuit (gate application only), one thread
    and the OpenMP restatement of the reference's parallel kernels on all host cores."""
    import torch

    import ruqu_b200 as rq
    from ruqu_b200 import workloads
    n, layers = 20, 40
    gates = workloads.random_layer_circuit(n, layers, 0)
    zs = [[(q, 3)] for q in range(n)]

    def run():
        st = rq.QuantumState(n, 0, "f64")
        st.apply_gates(gates)
        z = st.expectation_values(zs)
        bits = st.sample(4096, 42)
        return z, bits

    run()
    ms = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run()
        torch.cuda.synchronize()
        ms.append((time.perf_counter() - t0) * 1e3)
    S = (1 << n) * 16
    out = {"workload": "20 qubits, complex f64, 40 random layers (seed 0), <Z_i> x 20, 4096 shots",
           "ms": min(ms), "gates_per_s": len(gates) / (min(ms) / 1e3),
           "gbs_per_layer": (S + 2 * S * layers) / (min(ms) / 1e3) / 1e9}
    if with_cpu:
        import oracle
        o = oracle.OracleState(n, oracle.RQ_F64, 0)
        t0 = time.perf_counter()
        o.apply(gates)
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = {"ms": cpu_s * 1e3, "cores": 1, "kind": "port",
                               "sample": "the same %d gates on the oracle's scalar f64 reference kernels" % len(gates)}
        out["speedup_vs_cpu"] = cpu_s * 1e3 / min(ms)
        # the reference's parallel kernels (rayon, simd.rs:270-377) restated with OpenMP on all host cores
        o2 = oracle.OracleState(n, oracle.RQ_F64, 0)
        t0 = time.perf_counter()
        o2.apply(gates, parallel=True)
        par_s = time.perf_counter() - t0
        out["cpu_parallel"] = {"ms": par_s * 1e3, "cores": oracle.num_threads(), "kind": "port",
                               "sample": "the same gates on the oracle's OpenMP restatement of the reference's "
                                         "parallel kernels"}
        out["speedup_vs_cpu_parallel"] = par_s * 1e3 / min(ms)
    return out


def readout_leg(a, state, stream):
    """Read-out of the final state (the calls the reference's drivers make after a run):
    <Z_i> for every qubit (one FP64 reduction pass, state.rs:362-408), four two-qubit
    X/Y strings sharing one X/Y pattern (one paired pass) and 4096 shots
    (FP64 prefix tree + per-shot walks, the run_shots semantics of simulator.rs:107-147).
    Device time of each on the state's stream, and its HBM bytes: S for the <Z_i> pass;
    S read + 2^n x 8 B written for the tree's leaf level, then the fold levels."""
    import torch
    n = a.qubits
    S = (1 << n) * (8 if a.precision == "f32" else 16)
    zs = [[(q, 3)] for q in range(n)]
    xy = [[(0, 1), (1, 1)], [(0, 2), (1, 2)], [(0, 1), (1, 2)], [(0, 2), (1, 1)]]   # one X/Y pattern: one pass
    state.expectation_values(zs)
    state.expectation_values(xy)
    state.sample(16, 1)
    out = {}
    for name, fn in (("z_expectations", lambda: state.expectation_values(zs)),
                     ("xy_pair_expectations", lambda: state.expectation_values(xy)),
                     ("shots_4096", lambda: state.sample(4096, 7))):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        state.synchronize()
        out[name] = {"ms": e0.elapsed_time(e1)}
    out["z_expectations"]["gbs"] = S / (out["z_expectations"]["ms"] / 1e3) / 1e9
    out["xy_pair_expectations"]["gbs"] = S / (out["xy_pair_expectations"]["ms"] / 1e3) / 1e9
    tree = (1 << n) * 8
    out["shots_4096"]["tree_bytes"] = S + 2 * tree
    out["shots_4096"]["gbs"] = (S + 2 * tree) / (out["shots_4096"]["ms"] / 1e3) / 1e9
    return out


class _DeviceArray:
    """A raw device buffer seen by torch (__cuda_array_interface__), for measurements only."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "strides": None}


def _max_abs_diff(f32_state, f64_state, nq):
    import torch
    p32, _ = f32_state.device_pointer()
    p64, _ = f64_state.device_pointer()
    f32_state.synchronize()
    f64_state.synchronize()
    a = torch.as_tensor(_DeviceArray(p32, 2 << nq, "<f4"), device="cuda")
    b = torch.as_tensor(_DeviceArray(p64, 2 << nq, "<f8"), device="cuda")
    worst = 0.0
    chunk = 1 << 26
    for k in range(0, 2 << nq, chunk):
        worst = max(worst, float((a[k:k + chunk].double() - b[k:k + chunk]).abs().max()))
    return worst


def variants_leg(a, garr):
    """One timed run (after one warm-up run) of every execution mode on the benchmark circuit,
    and each f32 run's max-abs amplitude error against the complex f64 CUDA-core sweep."""
    import torch

    import ruqu_b200 as rq
    S = (1 << a.qubits) * 8
    layer_bytes = S + 2 * S * a.layers
    ref = rq.QuantumState(a.qubits, 0, "f64")
    ref.apply_gates(garr, rq.RQ_EXEC_SWEEP)
    ref.synchronize()
    out = {"value_bytes_per_run": layer_bytes, "reference": "complex f64 CUDA-core sweep of the same circuit"}
    for name, mode in (("unfused_per_gate", rq.RQ_EXEC_PER_GATE), ("sweep_cuda_cores", rq.RQ_EXEC_SWEEP),
                       ("tensor_core_3xtf32", rq.RQ_EXEC_SWEEP_TC), ("tensor_core_tf32", rq.RQ_EXEC_SWEEP_TC_FAST),
                       ("tensor_core_3xfp16", rq.RQ_EXEC_SWEEP_TC16)):
        st = rq.QuantumState(a.qubits, 0, "f32")
        plan = rq.Plan(st, garr, mode)
        _, sptr = st.device_pointer()
        stream = torch.cuda.ExternalStream(sptr)
        st.reset()
        plan.execute(st)
        st.reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.execute(st)
        e1.record(stream)
        st.synchronize()
        ms = e0.elapsed_time(e1)
        stats = plan.stats()
        out[name] = {"ms_per_circuit": ms, "gbs_per_layer": layer_bytes / (ms / 1e3) / 1e9,
                     "launches": stats["launches"], "sweeps": stats["sweeps"], "dense_ops": stats["dense_ops"],
                     "max_abs_vs_f64": _max_abs_diff(st, ref, a.qubits)}
        del plan
        del st
    del ref
    return out


def run_reference(a):
    """The reference arm: the oracle's OpenMP restatement of the reference's parallel
    kernels (one pass over the state per gate, the reference's execution model) on all host
    cores.  Each step times a bounded sample of the benchmark circuit (3 one-qubit gates and
    1 CNOT, in circuit order, each gate timed on its own); the circuit time is extrapolated
    from the per-kind mean gate times and the gate counts, and `value` is the GPU arm's
    per-layer byte count (S + 2S x layers) over that circuit time, so the two arms' values
    divide to the ratio of their circuit times.  Imports nothing that loads the CUDA library."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    import oracle
    from ruqu_b200 import workloads
    gates = workloads.random_layer_circuit(a.qubits, a.layers, a.seed)
    one, two = _gate_kinds(gates)
    prec = oracle.RQ_F32 if a.precision == "f32" else oracle.RQ_F64
    st = oracle.OracleState(a.qubits, prec, 0)
    S = (1 << a.qubits) * (8 if a.precision == "f32" else 16)
    layer_bytes = S + 2 * S * a.layers
    t1, t2, step_s = [], [], []
    for it in range(a.warmup + a.steps):
        _, timed, cores, st, (m1, m2) = cpu_circuit_time(a, True, 3, 1, st=st, start=it)
        if it >= a.warmup:
            t1.append(m1)
            t2.append(m2)
            step_s.append(timed)
    m1 = sum(t1) / len(t1)
    m2 = sum(t2) / len(t2)
    circuit_s = len(one) * m1 + len(two) * m2
    value = layer_bytes / circuit_s / 1e9
    cores = oracle.num_threads()
    sample = (f"per step 3 one-qubit gates and 1 CNOT of the {a.qubits}-qubit circuit on a {a.precision} state, "
              f"one pass over the state per gate (the reference's execution model), OpenMP restatement of the "
              f"reference's parallel kernels; circuit time extrapolated from the mean per-kind gate times "
              f"({m1 * 1e3:.1f} ms per 1q gate, {m2 * 1e3:.1f} ms per CNOT) x ({len(one)}, {len(two)}) gates")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * sum(step_s) / len(step_s), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": a.precision, "data": "synthetic",
        "config": {"workload": _workload_desc(a), "l2": "state larger than L2",
                   "value_bytes_per_circuit": layer_bytes, "circuit_ms": circuit_s * 1e3,
                   "circuit_ms_kind": "extrapolated from the timed gate sample",
                   "ms_per_step_is": "timed sample of 4 gates per step"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(a):
    import ctypes as C

    import numpy as np
    import torch

    import ruqu_b200 as rq
    from ruqu_b200 import workloads
    from ruqu_b200.circuit import gates_to_array

    ws, rank, local = _dist()
    dist = ws > 1
    if dist:
        from ruqu_b200 import dist as rqdist
        torch.cuda.set_device(local)
        tdist = rqdist.init("nccl", 120.0)
    rq.set_device(local)
    torch.cuda.set_device(local)

    mode = {"auto": rq.RQ_EXEC_AUTO, "per_gate": rq.RQ_EXEC_PER_GATE, "sweep": rq.RQ_EXEC_SWEEP,
            "tc": rq.RQ_EXEC_SWEEP_TC, "tc_fast": rq.RQ_EXEC_SWEEP_TC_FAST, "tc16": rq.RQ_EXEC_SWEEP_TC16}[a.mode]
    gates = workloads.random_layer_circuit(a.qubits, a.layers, a.seed)
    garr = gates_to_array(gates)
    state = rq.QuantumState(a.qubits, 0, a.precision)
    plan = rq.Plan(state, garr, mode)
    stats = plan.stats()
    elem = 8 if a.precision == "f32" else 16
    S = (1 << a.qubits) * elem
    step_bytes = S + stats["hbm_bytes"]
    _, sptr = state.device_pointer()
    stream = torch.cuda.ExternalStream(sptr, device=torch.device("cuda", local))

    def step(evs=None):
        # reset = one init kernel (stream-ordered, no host sync); the plan = the sweeps
        if evs:
            evs[0].record(stream)
        state.reset()
        if evs:
            evs[1].record(stream)
        plan.execute(state)
        if evs:
            evs[2].record(stream)

    for _ in range(a.warmup):
        step()
    state.synchronize()

    clocks = Clocks(local)
    if dist:
        tdist.barrier()
    torch.cuda.synchronize(local)
    state.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(a.steps)]
    for k in range(a.steps):
        step(ev[k])
    state.synchronize()
    torch.cuda.synchronize(local)
    clk = clocks.stop()
    total_ms = ev[0][0].elapsed_time(ev[-1][2])
    plan_ms = sum(e[1].elapsed_time(e[2]) for e in ev)
    init_ms = sum(e[0].elapsed_time(e[1]) for e in ev)
    if dist:
        total_ms = rqdist.max_over_ranks(total_ms)
    layer_bytes = S + 2 * S * a.layers          # |0> write + one read and write of the state per layer
    value = ws * layer_bytes * a.steps / (total_ms / 1e3) / 1e9
    peak, peak_kind = _peak()
    sweeps = max(1, stats["sweeps"] or stats["launches"])
    avg_launch_ms = plan_ms / (a.steps * sweeps)
    per_launch_bytes = (stats["hbm_bytes"] / sweeps)
    achieved = per_launch_bytes / (avg_launch_ms / 1e3) / 1e9

    # ---- end to end through the public API, host buffers ----
    e2e = None
    if not a.no_e2e:
        zs = [[(q, 3)] for q in range(a.qubits)]
        state.reset()
        state.apply_gates(garr, mode)
        state.expectation_values(zs)
        t0 = time.perf_counter()
        ksteps = max(1, min(a.steps, 3))
        for _ in range(ksteps):
            state.reset()
            state.apply_gates(garr, mode)
            state.expectation_values(zs)
        dt = (time.perf_counter() - t0) / ksteps
        e2e = {"value": ws * layer_bytes / dt / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": len(gates) * C.sizeof(rq._capi.RqGate),
               "d2h_bytes_per_step": 8 * a.qubits, "ms_per_step": dt * 1e3,
               "path": "QuantumState.reset + apply_gates(host list) + expectation_values(<Z_i>) -> host"}
        # the same path with a new angle set every step (what an optimizer's evaluations do):
        # the structure repeats, so each step rebuilds only the matrix tables and operand images
        vsteps = max(2, min(a.steps, 4))
        varr = [gates_to_array(workloads.random_layer_circuit(a.qubits, a.layers, 1000 + a.seed + k))
                for k in range(vsteps + 1)]
        state.reset()
        state.apply_gates(varr[0], mode)
        state.expectation_values(zs)
        t0 = time.perf_counter()
        for k in range(1, vsteps + 1):
            state.reset()
            state.apply_gates(varr[k], mode)
            state.expectation_values(zs)
        dtv = (time.perf_counter() - t0) / vsteps
        e2e["varying_angles"] = {"value": ws * layer_bytes / dtv / 1e9, "unit": UNIT, "ms_per_step": dtv * 1e3,
                                 "steps": vsteps, "ratio_to_e2e": dt / dtv,
                                 "path": "as e2e, with a new angle set (same gate structure) every step"}

    readout = None
    if not a.no_sampling:
        readout = readout_leg(a, state, stream)

    small = None
    if not a.no_small and rank == 0:
        small = small_circuit_leg(with_cpu=(ws == 1 and not a.no_cpu_baseline))

    variants = None
    if not a.no_variants and rank == 0:
        variants = variants_leg(a, garr)

    qaoa = None
    if not a.no_qaoa:
        qaoa = qaoa_batch_leg(a, ws, rank, with_cpu=(rank == 0 and ws == 1 and not a.no_cpu_baseline))
        if dist:
            qaoa["device_ms_max_over_ranks"] = rqdist.max_over_ranks(qaoa["device_ms"])
            qaoa["evals_per_s"] = a.qaoa_instances / (qaoa["device_ms_max_over_ranks"] / 1e3)

    vqe = None
    if not a.no_vqe:
        vqe = vqe_batch_leg(a, ws, rank, with_cpu=(rank == 0 and ws == 1 and not a.no_cpu_baseline))
        if dist:
            vqe["device_ms_max_over_ranks"] = rqdist.max_over_ranks(vqe["device_ms"])
            vqe["circuits_per_s"] = a.vqe_sets * 257 / (vqe["device_ms_max_over_ranks"] / 1e3)

    warm = None
    if not a.no_warm:
        warm = warmstart_leg(a, ws, rank, with_cpu=(rank == 0 and ws == 1 and not a.no_cpu_baseline))

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        v, circuit_s, secs, cores, desc = cpu_baseline_sample(a, parallel=False)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc, "seconds": secs,
               "circuit_ms": circuit_s * 1e3}

    if rank == 0:
        ref_layer_bytes = workloads.random_layer_bytes(a.qubits, a.layers, elem) + S
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": total_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": a.precision, "data": "synthetic",
            "config": {"workload": _workload_desc(a), "mode": a.mode, "parallelism": f"replicas x{ws}",
                       "l2": "state (%.1f GiB) larger than L2, no flush needed" % (S / 2**30),
                       "sweeps_per_step": stats["sweeps"], "launches_per_step": 1 + stats["launches"],
                       "phases_per_step": stats["phases"], "device_ops_per_step": stats["ops"],
                       "dense_tensor_core_ops_per_step": stats["dense_ops"],
                       "executed_as": _EXECUTED_AS.get(stats["exec_mode"], str(stats["exec_mode"])),
                       "local_qubits": stats["local_qubits"],
                       "value_bytes_per_step": layer_bytes, "plan_hbm_bytes_per_step": step_bytes,
                       "circuit_ms": total_ms / a.steps,
                       "layers_per_s": ws * a.layers * a.steps / (total_ms / 1e3),
                       "ms_init": init_ms / a.steps, "ms_gates": plan_ms / a.steps,
                       "unfused_reference_bytes_per_step": ref_layer_bytes},
            "roofline": {"bound": "hbm", "kernel": _KERNEL_OF.get(stats["exec_mode"], "k_sweep (multi-gate sweep)"),
                         "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "bytes_per_launch": per_launch_bytes, "avg_launch_ms": avg_launch_ms,
                         "traffic": _traffic_per_launch(a, stats)},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": a.steps * (1 + stats["launches"]),
            "readout": readout,
            "small_circuit": small,
            "variants": variants,
            "qaoa_batch": qaoa,
            "vqe_batch": vqe,
            "warm_start": warm,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    del plan
    del state
    if dist:
        tdist.barrier()
        tdist.destroy_process_group()


def main():
    a = _args()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
