"""Learned warm start for QAOA angles (rq_mlp_* of include/ruqu_cuda.h).

A small MLP maps label-free statistics of a graph (its size, edge density and
short-cycle counts, `cycle_features`) -- or, as an alternative encoding, the
padded adjacency (upper triangle of a 26-node adjacency matrix, 325 binary
features) -- to the 2p QAOA angles (gamma_1..gamma_p, beta_1..beta_p).  Its forward and backward
passes run on the GPU's BF16 tensor cores (tcgen05) with FP32 accumulation,
FP32 master weights and Adam on the device.  The reference has no learned
component; its run_qaoa starts every instance from gamma = beta = 0.5
(crates/ruqu-algorithms/src/qaoa.rs:221-222).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import lib
from .error import check

PAD_NODES = 26
FEATURES = PAD_NODES * (PAD_NODES - 1) // 2      # 325


def graph_features(n: int, edges, slots=None) -> np.ndarray:
    """Upper triangle (i < j, row-major) of the adjacency matrix padded to PAD_NODES nodes.
    slots (optional, n distinct values below PAD_NODES) places node v at row slots[v]."""
    if n > PAD_NODES:
        raise ValueError(f"graphs up to {PAD_NODES} nodes")
    pos = np.arange(n) if slots is None else np.asarray(slots)
    a = np.zeros((PAD_NODES, PAD_NODES), dtype=np.float32)
    for u, v in edges:
        a[pos[u], pos[v]] = a[pos[v], pos[u]] = 1.0
    iu = np.triu_indices(PAD_NODES, 1)
    return a[iu]


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    def __init__(self, n_in: int = FEATURES, h1: int = 256, h2: int = 256, n_out: int = 8, seed: int = 0):
        self.dims = (n_in, h1, h2, n_out)
        h = C.c_void_p()
        check(lib.rq_mlp_create(n_in, h1, h2, n_out, seed, C.byref(h)))
        self._h = h
        n = C.c_int64()
        check(lib.rq_mlp_num_params(self._h, C.byref(n)))
        self.nparam = n.value

    def get_params(self) -> np.ndarray:
        p = np.empty(self.nparam, dtype=np.float32)
        check(lib.rq_mlp_get_params(self._h, _fp(p)))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparam
        check(lib.rq_mlp_set_params(self._h, _fp(p)))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty((x.shape[0], self.dims[3]), dtype=np.float32)
        check(lib.rq_mlp_forward(self._h, _fp(x), x.shape[0], _fp(y)))
        return y

    def gradients(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.empty(self.nparam, dtype=np.float32)
        loss = C.c_float()
        check(lib.rq_mlp_gradients(self._h, _fp(x), _fp(t), x.shape[0], C.byref(loss), _fp(g)))
        return loss.value, g

    def train(self, x, t, batch: int = 256, steps: int = 100, lr: float = 1e-3) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        check(lib.rq_mlp_train(self._h, _fp(x), _fp(t), x.shape[0], batch, steps, lr, C.byref(loss)))
        return loss.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            lib.rq_mlp_destroy(h)
            self._h = None


def linear_ramp(p: int, delta: float = 0.75):
    """Plain start: gamma_l = -(l - 1/2)/p * delta, beta_l = (1 - (l - 1/2)/p) * delta, l = 1..p.

    The circuit of build_qaoa_circuit (qaoa.rs:125-153) applies Rzz(2 gamma) = exp(-i gamma ZZ)
    per edge, i.e. exp(+2i gamma cut(x)) up to a global phase, and Rx(2 beta) = exp(-i beta X):
    the expected cut rises from the random-guess |E|/2 for gamma < 0 with beta > 0, so the
    annealing-style ramp takes negative gammas."""
    f = (np.arange(1, p + 1) - 0.5) / p
    return -f * delta, (1.0 - f) * delta


N_CYCLE_FEATURES = 7


def cycle_features(graphs) -> np.ndarray:
    """Label-free graph statistics, one row per graph: n / 26, edges per node, mean degree,
    and tr(A^k) / (2 k n) for k = 3..6 (closed walks of length k per node; tr(A^3) / 6 is
    the triangle count).  Optimal QAOA angles of graphs of one size vary with their short
    cycles (on 12-node 3-regular graphs, triangle and 4-cycle counts alone explain 26-70 %
    of the variance of the optimal angles around their mean)."""
    out = np.zeros((len(graphs), N_CYCLE_FEATURES))
    for gi, (n, edges) in enumerate(graphs):
        a = np.zeros((n, n))
        for u, v in edges:
            a[u, v] = a[v, u] = 1.0
        row = [n / PAD_NODES, len(edges) / max(n, 1), a.sum() / max(n, 1)]
        ak = a @ a
        for k in range(3, 7):
            ak = ak @ a
            row.append(np.trace(ak) / (2 * k * max(n, 1)))
        out[gi] = row
    return out


def features(graphs, copies: int = 1, seed=None) -> np.ndarray:
    """Feature rows of the graphs.  With a seed, each graph gives `copies` rows, each
    with its nodes placed at random distinct rows of the padded matrix (graph-major
    order): the angles do not depend on node labels, and every input position is
    exercised during training whatever the graph sizes."""
    for n, _ in graphs:
        if n > PAD_NODES:
            raise ValueError(f"graphs up to {PAD_NODES} nodes")
    nrows = len(graphs) * (copies if seed is not None else 1)
    if seed is None:
        pos = np.tile(np.arange(PAD_NODES), (nrows, 1))
    else:   # a random placement per row: the first n entries of a random permutation
        pos = np.argsort(np.random.default_rng(seed).random((nrows, PAD_NODES)), axis=1)
    reps = copies if seed is not None else 1
    row_of, us, vs = [], [], []
    for gi, (n, edges) in enumerate(graphs):
        if not len(edges):
            continue
        e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
        for c in range(reps):
            r = gi * reps + c
            row_of.append(np.full(len(e), r))
            us.append(pos[r, e[:, 0]])
            vs.append(pos[r, e[:, 1]])
    a = np.zeros((nrows, PAD_NODES, PAD_NODES), dtype=np.float32)
    if row_of:
        rr, uu, vv = np.concatenate(row_of), np.concatenate(us), np.concatenate(vs)
        a[rr, uu, vv] = 1.0
        a[rr, vv, uu] = 1.0
    iu = np.triu_indices(PAD_NODES, 1)
    return np.ascontiguousarray(a[:, iu[0], iu[1]])


class WarmStart:
    """Learned QAOA warm start: an Mlp from graph features to the 2p angles.

    Optimal QAOA angles of one graph family concentrate around a size-dependent value, so
    the prediction is trend(n) + sd * MLP(adjacency): trend(n) is the training set's mean
    angle vector for graphs of n nodes (a straight line in n, fitted to the per-size means,
    for sizes not seen in training) and the network learns the per-graph correction, in
    units of the residual spread sd.  An untrained network (or one that never beats zero on
    the held-out slice) predicts the trend alone -- the "mean predictor", which
    mean_angles() returns for comparison.  With the cycle encoding each graph gives one
    row of standardised cycle statistics; with the adjacency encoding training rows place
    each graph's nodes at random rows of the padded matrix (`copies` placements per graph)
    and predictions average `tta` placements.  A held-out slice of the graphs picks the
    parameters with the lowest validation error."""

    def __init__(self, p: int, hidden: int = 256, seed: int = 5, encoding: str = "adjacency"):
        """encoding: "cycles" feeds the network the standardised label-free statistics of
        cycle_features (in the first inputs, the rest zero); "adjacency" the padded
        adjacency of randomly placed nodes."""
        if encoding not in ("cycles", "adjacency"):
            raise ValueError("encoding is 'cycles' or 'adjacency'")
        self.p = p
        self.encoding = encoding
        self.fmean = np.zeros(N_CYCLE_FEATURES)
        self.fstd = np.ones(N_CYCLE_FEATURES)
        self.net = Mlp(h1=hidden, h2=hidden, n_out=2 * p, seed=seed)
        self.sd = np.ones(2 * p)
        self.size_mean = {}                 # n -> mean angle vector of the training graphs of size n
        self.line = np.zeros((2, 2 * p))    # trend(n) = line[0] + line[1] * n for unseen sizes
        self.precond = {}

    def _rows(self, graphs, copies: int, seed) -> np.ndarray:
        """Network input rows: `copies` random placements per graph (adjacency), or one row
        of standardised cycle statistics per graph repeated `copies` times (cycles)."""
        if self.encoding == "adjacency":
            return features(graphs, copies, seed=seed)
        z = (cycle_features(graphs) - self.fmean) / self.fstd
        x = np.zeros((len(graphs), FEATURES), dtype=np.float32)
        x[:, :N_CYCLE_FEATURES] = z
        return np.ascontiguousarray(np.repeat(x, copies, axis=0))

    def trend(self, ns) -> np.ndarray:
        """Mean angle vector for graphs of each size in ns (seen sizes: their training mean;
        others: the least-squares line through the per-size means)."""
        return np.stack([self.size_mean[int(n)] if int(n) in self.size_mean else self.line[0] + self.line[1] * n
                         for n in ns])

    def mean_angles(self, graphs):
        """The mean predictor: trend(n) for each graph (gammas, betas)."""
        y = self.trend([n for n, _ in graphs])
        return y[:, :self.p], y[:, self.p:]

    def fit(self, graphs, gammas, betas, copies: int = 4, val_fraction: float = 0.125, chunks: int = 12,
            chunk_steps: int = 500, lr: float = 1e-3, batch: int = 256, seed: int = 3) -> list:
        """Returns the validation error after each training chunk, as a fraction of the
        residual variance (below 1: the network predicts part of the per-graph correction)."""
        y = np.concatenate([np.asarray(gammas, dtype=np.float64), np.asarray(betas, dtype=np.float64)], axis=1)
        nval = max(1, int(len(graphs) * val_fraction))
        ntr = len(graphs) - nval
        ns = np.array([n for n, _ in graphs])
        sizes = sorted(set(ns[:ntr].tolist()))
        self.size_mean = {n: y[:ntr][ns[:ntr] == n].mean(axis=0) for n in sizes}
        if len(sizes) > 1:
            A = np.stack([np.ones(len(sizes)), np.array(sizes, dtype=np.float64)], axis=1)
            self.line = np.linalg.lstsq(A, np.stack([self.size_mean[n] for n in sizes]), rcond=None)[0]
        else:
            self.line = np.stack([self.size_mean[sizes[0]], np.zeros(2 * self.p)])
        r = y - self.trend(ns)
        # residual spreads below 1e-3 rad carry no information for the optimizer and are not
        # blown up to unit variance
        self.sd = np.maximum(r[:ntr].std(axis=0), 1e-3)
        z = r / self.sd
        if self.encoding == "cycles":   # statistics of the training graphs set the scaling
            copies = 1
            f = cycle_features(graphs[:ntr])
            self.fmean = f.mean(axis=0)
            sd = f.std(axis=0)
            self.fstd = np.where(sd > 1e-9, sd, 1.0)
        x = self._rows(graphs[:ntr], copies, seed)
        t = np.repeat(z[:ntr], copies, axis=0).astype(np.float32)
        xv = self._rows(graphs[ntr:], copies, seed + 1)
        tv = np.repeat(z[ntr:], copies, axis=0).astype(np.float32)
        var = float(np.mean(tv.astype(np.float64) ** 2))
        best, best_p, hist = var, None, []
        for c in range(chunks):
            self.net.train(x, t, batch=batch, steps=chunk_steps, lr=lr if c < (2 * chunks) // 3 else lr / 3)
            vl = float(np.mean((self.net.forward(xv) - tv) ** 2)) / max(var, 1e-30)
            hist.append(vl)
            if not np.isfinite(vl):     # diverged: keep the best parameters seen so far
                break
            if vl * var < best:
                best, best_p = vl * var, self.net.get_params()
        if best_p is None:     # never better than the mean: predict the mean
            self.net.set_params(np.zeros(self.net.nparam, dtype=np.float32))
        else:
            self.net.set_params(best_p)
        return hist

    def fit_curvature(self, graphs, gammas, betas, h: float = 1e-3, max_graphs: int = 512) -> dict:
        """Learn the curvature of the energy landscape near the optimum: for each graph size n,
        the average Hessian of <C> at the training graphs' optimised angles (central
        differences, step h, of exact adjoint gradients on the GPU), stored as the ascent
        preconditioner P_n = -H_n^-1 (eigenvalues clamped to keep -H positive definite).
        Returns {n: eigenvalues of H_n}."""
        from .batch import QaoaBatch
        th = np.concatenate([np.asarray(gammas, dtype=np.float64), np.asarray(betas, dtype=np.float64)], axis=1)
        sub = np.arange(min(len(graphs), max_graphs))
        qb = QaoaBatch([graphs[i] for i in sub], self.p, "f32")
        cols = []
        for j in range(2 * self.p):
            tp, tm = th[sub].copy(), th[sub].copy()
            tp[:, j] += h
            tm[:, j] -= h
            _, gp = qb.gradient(tp[:, :self.p], tp[:, self.p:])
            _, gm = qb.gradient(tm[:, :self.p], tm[:, self.p:])
            cols.append((gp - gm) / (2 * h))
        H = np.stack(cols, axis=2)
        H = 0.5 * (H + H.transpose(0, 2, 1))
        ns = np.array([graphs[i][0] for i in sub])
        self.precond = {}
        eig = {}
        for n in sorted(set(ns.tolist())):
            Hn = H[ns == n].mean(axis=0)
            w, V = np.linalg.eigh(Hn)
            eig[n] = w
            w = np.minimum(w, -1e-3 * max(1.0, float(np.max(np.abs(w)))))
            self.precond[n] = (V * (-1.0 / w)) @ V.T
        return eig

    def preconditioners(self, graphs) -> np.ndarray:
        """P_n of each graph's size (the nearest learned size when n was not seen)."""
        sizes = np.array(sorted(self.precond))
        return np.stack([self.precond[int(sizes[np.argmin(np.abs(sizes - n))])] for n, _ in graphs])

    def predict(self, graphs, tta: int = 8, seed: int = 9):
        if self.encoding == "cycles":
            tta = 1
        x = self._rows(graphs, tta, seed)
        z = self.net.forward(x).reshape(len(graphs), tta, -1).mean(axis=1).astype(np.float64)
        y = self.trend([n for n, _ in graphs]) + self.sd * z
        return y[:, :self.p], y[:, self.p:]

