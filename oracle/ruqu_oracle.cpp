// ruqu_oracle.cpp -- CPU oracle for the ruqu-core state-vector path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in C++, the semantics of the
// reference's scalar f64 / f32 state-vector engine so that the CUDA library can
// be checked against it.  Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline / reference legs may load it; the product library never does.
//
// The reference is Rust and cannot be compiled in this environment (no cargo,
// no rustc), so the oracle is a restatement, pinned against the known-answer
// tests of crates/ruqu-core/tests/*.rs and crates/ruqu-algorithms/tests/*.rs
// (ported in tests/test_oracle_kats.py).  The measurement RNG of the reference
// (rand 0.8.6 StdRng = ChaCha12 from rand_chacha 0.3.1, seeded through
// rand_core 0.6.4 seed_from_u64) is third-party and no reference test pins a
// concrete draw, so draws are taken from the documented Philox4x32-10 stream
// that the CUDA library also uses: exact agreement with the Rust binary's
// random draws is "parity unpinned"; everything else is pinned.
//
// Floating-point order follows the reference: complex product
// (a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re) (types.rs:80-89), matrix-
// vector rows summed left to right (state.rs:225-226, 268-272).  Build with
// -ffp-contract=off so no FMA contraction changes the rounding.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include <random>
#include <stdexcept>
#include <string>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/ruqu_cuda.h"

namespace {

// ---------------------------------------------------------------------------
// Complex types (types.rs:8-180, mixed_precision.rs:24-160)
// ---------------------------------------------------------------------------
template <typename R>
struct Cx {
    R re, im;
};
template <typename R>
inline Cx<R> cadd(Cx<R> a, Cx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <typename R>
inline Cx<R> cmul(Cx<R> a, Cx<R> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R>
inline Cx<R> cscale(Cx<R> a, R s) { return {a.re * s, a.im * s}; }
template <typename R>
inline Cx<R> cconj(Cx<R> a) { return {a.re, -a.im}; }
template <typename R>
inline R cnorm_sq(Cx<R> a) { return a.re * a.re + a.im * a.im; }

using C64 = Cx<double>;
using C32 = Cx<float>;

inline C64 from_polar(double r, double theta) { return {r * std::cos(theta), r * std::sin(theta)}; }

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11).  Round function: two 32x32->64 multiplies with
// the published multipliers, Weyl key schedule with the published constants.
// ---------------------------------------------------------------------------
struct U4 { uint32_t v[4]; };

inline U4 philox(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k0 += W0; k1 += W1; }
        uint64_t p0 = (uint64_t)M0 * c.v[0];
        uint64_t p1 = (uint64_t)M1 * c.v[2];
        U4 n;
        n.v[0] = (uint32_t)(p1 >> 32) ^ c.v[1] ^ k0;
        n.v[1] = (uint32_t)p1;
        n.v[2] = (uint32_t)(p0 >> 32) ^ c.v[3] ^ k1;
        n.v[3] = (uint32_t)p0;
        c = n;
    }
    return c;
}

// Draw `index` of stream `stream` under key `seed`: counter
// (lo32(index/2), hi32(index/2), stream, 0); even draws take words (0,1),
// odd draws words (2,3); the 64-bit word hi<<32|lo keeps its top 53 bits.
inline double uniform(uint64_t seed, uint32_t stream, uint64_t index) {
    uint64_t blk = index >> 1;
    U4 c{{(uint32_t)blk, (uint32_t)(blk >> 32), stream, 0u}};
    U4 x = philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint32_t hi = (index & 1) ? x.v[2] : x.v[0];
    uint32_t lo = (index & 1) ? x.v[3] : x.v[1];
    uint64_t w = ((uint64_t)hi << 32) | lo;
    return (double)(w >> 11) * (1.0 / 9007199254740992.0);
}

// ---------------------------------------------------------------------------
// Gate matrices (gate.rs:72-198)
// ---------------------------------------------------------------------------
using M2 = C64[2][2];
using M4 = C64[4][4];

const double FRAC_1_SQRT_2 = 0.70710678118654752440;

bool matrix_1q(const rq_gate& g, M2 m) {
    const C64 c0{0, 0}, c1{1, 0}, ci{0, 1};
    auto set = [&](C64 a, C64 b, C64 c, C64 d) { m[0][0] = a; m[0][1] = b; m[1][0] = c; m[1][1] = d; };
    switch (g.kind) {
        case RQ_GATE_H: { C64 h{FRAC_1_SQRT_2, 0}; set(h, h, h, {-h.re, -h.im}); return true; }
        case RQ_GATE_X: set(c0, c1, c1, c0); return true;
        case RQ_GATE_Y: set(c0, {-ci.re, -ci.im}, ci, c0); return true;
        case RQ_GATE_Z: set(c1, c0, c0, {-c1.re, -c1.im}); return true;
        case RQ_GATE_S: set(c1, c0, c0, ci); return true;
        case RQ_GATE_SDG: set(c1, c0, c0, {-ci.re, -ci.im}); return true;
        case RQ_GATE_T: set(c1, c0, c0, {FRAC_1_SQRT_2, FRAC_1_SQRT_2}); return true;
        case RQ_GATE_TDG: set(c1, c0, c0, {FRAC_1_SQRT_2, -FRAC_1_SQRT_2}); return true;
        case RQ_GATE_RX: {
            double half = g.angle / 2.0;
            C64 c{std::cos(half), 0.0}, s{0.0, -std::sin(half)};
            set(c, s, s, c); return true;
        }
        case RQ_GATE_RY: {
            double half = g.angle / 2.0;
            double ch = std::cos(half), sh = std::sin(half);
            set({ch, 0}, {-sh, 0}, {sh, 0}, {ch, 0}); return true;
        }
        case RQ_GATE_RZ: {
            double half = g.angle / 2.0;
            set(from_polar(1.0, -half), c0, c0, from_polar(1.0, half)); return true;
        }
        case RQ_GATE_PHASE: set(c1, c0, c0, from_polar(1.0, g.angle)); return true;
        case RQ_GATE_UNITARY1Q:
            set({g.m[0], g.m[1]}, {g.m[2], g.m[3]}, {g.m[4], g.m[5]}, {g.m[6], g.m[7]});
            return true;
        default: return false;
    }
}

bool matrix_2q(const rq_gate& g, M4 m) {
    const C64 c0{0, 0}, c1{1, 0};
    for (int r = 0; r < 4; ++r) for (int c = 0; c < 4; ++c) m[r][c] = c0;
    switch (g.kind) {
        case RQ_GATE_CNOT: m[0][0] = c1; m[1][1] = c1; m[2][3] = c1; m[3][2] = c1; return true;
        case RQ_GATE_CZ: m[0][0] = c1; m[1][1] = c1; m[2][2] = c1; m[3][3] = {-1.0, -0.0}; return true;
        case RQ_GATE_SWAP: m[0][0] = c1; m[1][2] = c1; m[2][1] = c1; m[3][3] = c1; return true;
        case RQ_GATE_RZZ: {
            double half = g.angle / 2.0;
            C64 en = from_polar(1.0, -half), ep = from_polar(1.0, half);
            m[0][0] = en; m[1][1] = ep; m[2][2] = ep; m[3][3] = en; return true;
        }
        default: return false;
    }
}

bool is_2q(int k) { return k == RQ_GATE_CNOT || k == RQ_GATE_CZ || k == RQ_GATE_SWAP || k == RQ_GATE_RZZ; }
bool is_non_unitary(int k) { return k == RQ_GATE_MEASURE || k == RQ_GATE_RESET || k == RQ_GATE_BARRIER; }

thread_local std::string g_err;

// ---------------------------------------------------------------------------
// State (state.rs:18-450 for R=double, mixed_precision.rs:193-549 for float)
// ---------------------------------------------------------------------------
struct StateBase {
    virtual ~StateBase() {}
    uint32_t nq = 0;
    uint64_t seed = 0;
    uint64_t draws = 0;
    std::vector<rq_measurement> record;
    double next_uniform() { return uniform(seed, 0, draws++); }
};

template <typename R>
struct State : StateBase {
    std::vector<Cx<R>> a;

    void init(uint32_t n) {
        nq = n;
        a.assign((size_t)1 << n, Cx<R>{0, 0});
        a[0] = Cx<R>{1, 0};
    }

    static Cx<R> cvt(C64 c) { return {(R)c.re, (R)c.im}; }

    // state.rs:214-229
    void apply_1q(uint32_t q, const M2 md) {
        Cx<R> m[2][2];
        for (int r = 0; r < 2; ++r) for (int c = 0; c < 2; ++c) m[r][c] = cvt(md[r][c]);
        size_t step = (size_t)1 << q, n = a.size();
        for (size_t bs = 0; bs < n; bs += step << 1) {
            for (size_t i = bs; i < bs + step; ++i) {
                size_t j = i + step;
                Cx<R> x = a[i], y = a[j];
                a[i] = cadd(cmul(m[0][0], x), cmul(m[0][1], y));
                a[j] = cadd(cmul(m[1][0], x), cmul(m[1][1], y));
            }
        }
    }

    // state.rs:238-276 (the full base loop with its 3/4 skip)
    void apply_2q(uint32_t q1, uint32_t q2, const M4 md) {
        Cx<R> m[4][4];
        for (int r = 0; r < 4; ++r) for (int c = 0; c < 4; ++c) m[r][c] = cvt(md[r][c]);
        size_t b1 = (size_t)1 << q1, b2 = (size_t)1 << q2, n = a.size();
        for (size_t base = 0; base < n; ++base) {
            if ((base & b1) || (base & b2)) continue;
            size_t idx[4] = {base, base | b2, base | b1, base | b1 | b2};
            Cx<R> v[4] = {a[idx[0]], a[idx[1]], a[idx[2]], a[idx[3]]};
            for (int r = 0; r < 4; ++r) {
                Cx<R> acc = cmul(m[r][0], v[0]);
                acc = cadd(acc, cmul(m[r][1], v[1]));
                acc = cadd(acc, cmul(m[r][2], v[2]));
                acc = cadd(acc, cmul(m[r][3], v[3]));
                a[idx[r]] = acc;
            }
        }
    }

    // OpenMP restatement of the reference's rayon kernels (simd.rs:270-377);
    // used only for the multi-core CPU timing, never for parity.
    void apply_1q_par(uint32_t q, const M2 md) {
        Cx<R> m[2][2];
        for (int r = 0; r < 2; ++r) for (int c = 0; c < 2; ++c) m[r][c] = cvt(md[r][c]);
        size_t step = (size_t)1 << q, half = a.size() >> 1;
        Cx<R>* A = a.data();
#pragma omp parallel for schedule(static)
        for (size_t p = 0; p < half; ++p) {
            size_t i = ((p >> q) << (q + 1)) | (p & (step - 1));
            size_t j = i + step;
            Cx<R> x = A[i], y = A[j];
            A[i] = cadd(cmul(m[0][0], x), cmul(m[0][1], y));
            A[j] = cadd(cmul(m[1][0], x), cmul(m[1][1], y));
        }
    }
    void apply_2q_par(uint32_t q1, uint32_t q2, const M4 md) {
        Cx<R> m[4][4];
        for (int r = 0; r < 4; ++r) for (int c = 0; c < 4; ++c) m[r][c] = cvt(md[r][c]);
        size_t b1 = (size_t)1 << q1, b2 = (size_t)1 << q2, quarter = a.size() >> 2;
        uint32_t lo = std::min(q1, q2), hi = std::max(q1, q2);
        Cx<R>* A = a.data();
#pragma omp parallel for schedule(static)
        for (size_t g = 0; g < quarter; ++g) {
            size_t base = ((g >> lo) << (lo + 1)) | (g & (((size_t)1 << lo) - 1));
            base = ((base >> hi) << (hi + 1)) | (base & (((size_t)1 << hi) - 1));
            size_t idx[4] = {base, base | b2, base | b1, base | b1 | b2};
            Cx<R> v[4] = {A[idx[0]], A[idx[1]], A[idx[2]], A[idx[3]]};
            for (int r = 0; r < 4; ++r) {
                Cx<R> acc = cmul(m[r][0], v[0]);
                acc = cadd(acc, cmul(m[r][1], v[1]));
                acc = cadd(acc, cmul(m[r][2], v[2]));
                acc = cadd(acc, cmul(m[r][3], v[3]));
                A[idx[r]] = acc;
            }
        }
    }

    // state.rs:288-326 (f64) / mixed_precision.rs:470-507 (f32: p0 summed in f32)
    rq_measurement measure(uint32_t q) {
        size_t bit = (size_t)1 << q, n = a.size();
        R p0 = 0;
        for (size_t i = 0; i < n; ++i)
            if (!(i & bit)) p0 += cnorm_sq(a[i]);
        double u = next_uniform();
        bool result = u >= (double)p0;
        R prob = result ? (R)1 - p0 : p0;
        R nf = prob > 0 ? (R)1 / std::sqrt(prob) : (R)0;
        for (size_t i = 0; i < n; ++i) {
            bool one = (i & bit) != 0;
            a[i] = (one == result) ? cscale(a[i], nf) : Cx<R>{0, 0};
        }
        rq_measurement m{q, result ? 1 : 0, (double)prob};
        record.push_back(m);
        return m;
    }

    // state.rs:343-352
    void reset_qubit(uint32_t q) {
        rq_measurement m = measure(q);
        if (m.result) {
            rq_gate x{}; x.kind = RQ_GATE_X; x.q0 = q;
            M2 mx; matrix_1q(x, mx);
            apply_1q(q, mx);
        }
    }

    // state.rs:123-137
    double prob_qubit(uint32_t q) const {
        size_t bit = (size_t)1 << q;
        double p1 = 0.0;
        for (size_t i = 0; i < a.size(); ++i)
            if (i & bit) p1 += (double)cnorm_sq(a[i]);
        return p1;
    }

    // state.rs:362-400 (for f32 states the amplitudes are widened to f64
    // first, which is what QuantumStateF32::to_f64 + expectation_value does)
    double expectation(const rq_pauli_op* ops, uint32_t nops) const {
        C64 result{0, 0};
        size_t n = a.size();
        for (size_t i = 0; i < n; ++i) {
            size_t j = i;
            C64 phase{1, 0};
            for (uint32_t k = 0; k < nops; ++k) {
                uint32_t q = ops[k].qubit;
                size_t bit = (i >> q) & 1;
                switch (ops[k].op) {
                    case RQ_PAULI_X: j ^= (size_t)1 << q; break;
                    case RQ_PAULI_Y:
                        j ^= (size_t)1 << q;
                        phase = bit == 0 ? cmul(phase, C64{0, 1}) : cmul(phase, C64{0, -1});
                        break;
                    case RQ_PAULI_Z:
                        if (bit == 1) phase = C64{-phase.re, -phase.im};
                        break;
                    default: break;
                }
            }
            C64 aj{(double)a[j].re, (double)a[j].im}, ai{(double)a[i].re, (double)a[i].im};
            result = cadd(result, cmul(cmul(cconj(aj), phase), ai));
        }
        return result.re;
    }

    // state.rs:415-423
    void normalize() {
        double ns = 0.0;
        for (auto& x : a) ns += (double)cnorm_sq(x);
        if (ns > 0.0) {
            double inv = 1.0 / std::sqrt(ns);
            for (auto& x : a) x = Cx<R>{(R)(x.re * inv), (R)(x.im * inv)};
        }
    }
};

std::vector<double> probs_of(const StateBase* s) {
    if (auto d = dynamic_cast<const State<double>*>(s)) {
        std::vector<double> p(d->a.size());
        for (size_t i = 0; i < p.size(); ++i) p[i] = cnorm_sq(d->a[i]);
        return p;
    }
    auto f = dynamic_cast<const State<float>*>(s);
    std::vector<double> p(f->a.size());
    for (size_t i = 0; i < p.size(); ++i) p[i] = (double)cnorm_sq(f->a[i]);  // f32 norm, widened (mixed_precision.rs:282-284)
    return p;
}

template <typename R>
int apply_gate_impl(State<R>* s, const rq_gate& g, std::vector<rq_measurement>* outs, bool par) {
    // validation (state.rs:160-162, 179-184)
    uint32_t qs[2]; int nq = 0;
    if (g.kind == RQ_GATE_BARRIER) nq = 0;
    else if (is_2q(g.kind)) { qs[0] = g.q0; qs[1] = g.q1; nq = 2; }
    else { qs[0] = g.q0; nq = 1; }
    for (int k = 0; k < nq; ++k)
        if (qs[k] >= s->nq) {
            g_err = "invalid qubit index " + std::to_string(qs[k]) + " for " + std::to_string(s->nq) + "-qubit system";
            return RQ_ERR_INVALID_QUBIT_INDEX;
        }
    switch (g.kind) {
        case RQ_GATE_BARRIER: return RQ_OK;
        case RQ_GATE_MEASURE: { auto m = s->measure(g.q0); if (outs) outs->push_back(m); return RQ_OK; }
        case RQ_GATE_RESET: s->reset_qubit(g.q0); return RQ_OK;
        default: break;
    }
    if (is_2q(g.kind)) {
        if (g.q0 == g.q1) {
            g_err = "circuit error: two-qubit gate requires distinct qubits, got " + std::to_string(g.q0) + " and " + std::to_string(g.q1);
            return RQ_ERR_CIRCUIT;
        }
        M4 m; matrix_2q(g, m);
        if (par) s->apply_2q_par(g.q0, g.q1, m); else s->apply_2q(g.q0, g.q1, m);
        return RQ_OK;
    }
    M2 m;
    if (!matrix_1q(g, m)) { g_err = "circuit error: unsupported gate"; return RQ_ERR_CIRCUIT; }
    if (par) s->apply_1q_par(g.q0, m); else s->apply_1q(g.q0, m);
    return RQ_OK;
}

int check_qubits(uint32_t nq, int prec) {
    uint32_t maxq = prec == RQ_F32 ? RQ_MAX_QUBITS_F32 : RQ_MAX_QUBITS_F64;
    if (nq == 0) { g_err = "circuit error: cannot create quantum state with 0 qubits"; return RQ_ERR_CIRCUIT; }
    if (nq > maxq) {
        g_err = "qubit limit exceeded: requested " + std::to_string(nq) + ", maximum " + std::to_string(maxq);
        return RQ_ERR_QUBIT_LIMIT_EXCEEDED;
    }
    return RQ_OK;
}

// Prefix-tree sampler over the measured qubits, in measurement order:
// level k holds the mass of every k-bit outcome prefix; p0 at step k is
// mass(prefix,0) / (mass(prefix,0) + mass(prefix,1)).  Mathematically equal
// to the reference's collapse-and-renormalise loop (state.rs:288-335) run
// once per shot; orc_run_shots_literal checks the equality at small n.
void tree_sample(const double* p, uint32_t n, const uint32_t* qs, uint32_t m,
                 uint64_t base_seed, uint64_t shots, uint64_t* out) {
    // bit position of each qubit in the permuted index: measured qubits first
    // (in order, first occurrence), then the unmeasured ones ascending.
    std::vector<int> pos(n, -1);
    std::vector<uint32_t> order;  // permuted position -> qubit
    for (uint32_t k = 0; k < m; ++k)
        if (pos[qs[k]] < 0) { pos[qs[k]] = (int)order.size(); order.push_back(qs[k]); }
    uint32_t md = (uint32_t)order.size();
    for (uint32_t q = 0; q < n; ++q)
        if (pos[q] < 0) { pos[q] = (int)order.size(); order.push_back(q); }
    size_t N = (size_t)1 << n;
    std::vector<double> lvl(N);
    for (size_t i = 0; i < N; ++i) {
        size_t j = 0;
        for (uint32_t q = 0; q < n; ++q) j |= ((i >> q) & 1) << pos[q];
        lvl[j] = p[i];
    }
    // fold levels n -> 0; keep levels 0..md
    std::vector<std::vector<double>> L(md + 1);
    std::vector<double> cur = lvl;
    for (int k = (int)n; k >= 0; --k) {
        if ((uint32_t)k <= md) L[k] = cur;
        if (k == 0) break;
        size_t h = (size_t)1 << (k - 1);
        std::vector<double> nxt(h);
        for (size_t j = 0; j < h; ++j) nxt[j] = cur[j] + cur[j + h];
        cur.swap(nxt);
    }
    for (uint64_t s = 0; s < shots; ++s) {
        uint64_t key = base_seed + s;
        size_t prefix = 0;
        uint64_t bits = 0;
        std::vector<int> outcome(n, -1);
        for (uint32_t k = 0; k < m; ++k) {
            double u = uniform(key, 0, k);
            uint32_t q = qs[k];
            int r;
            if (outcome[q] >= 0) {
                r = outcome[q];  // repeated measurement of a collapsed qubit
            } else {
                uint32_t lev = (uint32_t)pos[q];  // == number of bits already fixed
                double m0 = L[lev + 1][prefix];
                double m1 = L[lev + 1][prefix | ((size_t)1 << lev)];
                double p0 = m0 / (m0 + m1);
                r = u >= p0 ? 1 : 0;
                prefix |= (size_t)r << lev;
                outcome[q] = r;
            }
            if (r) bits |= (uint64_t)1 << q; else bits &= ~((uint64_t)1 << q);
        }
        out[s] = bits;
    }
}

template <typename R>
State<R>* as(StateBase* s) { return dynamic_cast<State<R>*>(s); }

}  // namespace

// ===========================================================================
// C ABI for the Python test harness (ctypes)
// ===========================================================================
extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
    U4 c{{ctr[0], ctr[1], ctr[2], ctr[3]}};
    U4 x = philox(c, key[0], key[1]);
    for (int i = 0; i < 4; ++i) out[i] = x.v[i];
}

double orc_uniform(uint64_t seed, uint32_t stream, uint64_t index) { return uniform(seed, stream, index); }

int orc_state_new(uint32_t nq, int32_t prec, uint64_t seed, int32_t seeded, void** out) {
    int rc = check_qubits(nq, prec);
    if (rc) return rc;
    StateBase* s;
    if (prec == RQ_F32) { auto* f = new State<float>(); f->init(nq); s = f; }
    else { auto* d = new State<double>(); d->init(nq); s = d; }
    s->seed = seeded ? seed : std::random_device{}();
    *out = s;
    return RQ_OK;
}

int orc_state_from_amplitudes(const double* amps, uint64_t len, uint32_t nq, int32_t prec, uint64_t seed, void** out) {
    uint32_t maxq = prec == RQ_F32 ? RQ_MAX_QUBITS_F32 : RQ_MAX_QUBITS_F64;
    if (nq > maxq) { g_err = "qubit limit exceeded"; return RQ_ERR_QUBIT_LIMIT_EXCEEDED; }
    if (len != ((uint64_t)1 << nq)) {
        g_err = "invalid state vector: length " + std::to_string(len) + " does not match 2^" + std::to_string(nq);
        return RQ_ERR_INVALID_STATE_VECTOR;
    }
    StateBase* s;
    if (prec == RQ_F32) {
        auto* f = new State<float>(); f->nq = nq; f->a.resize(len);
        for (size_t i = 0; i < len; ++i) f->a[i] = {(float)amps[2 * i], (float)amps[2 * i + 1]};
        s = f;
    } else {
        auto* d = new State<double>(); d->nq = nq; d->a.resize(len);
        for (size_t i = 0; i < len; ++i) d->a[i] = {amps[2 * i], amps[2 * i + 1]};
        s = d;
    }
    s->seed = seed;
    *out = s;
    return RQ_OK;
}

void orc_state_free(void* s) { delete (StateBase*)s; }

int orc_apply(void* h, const rq_gate* gates, uint64_t n, rq_measurement* out, uint64_t cap, uint64_t* nout, int32_t parallel) {
    StateBase* s = (StateBase*)h;
    std::vector<rq_measurement> outs;
    for (uint64_t k = 0; k < n; ++k) {
        int rc;
        if (auto d = as<double>(s)) rc = apply_gate_impl(d, gates[k], &outs, parallel != 0);
        else rc = apply_gate_impl(as<float>(s), gates[k], &outs, parallel != 0);
        if (rc) return rc;
    }
    if (nout) *nout = outs.size();
    for (size_t k = 0; k < outs.size() && k < cap; ++k) out[k] = outs[k];
    return RQ_OK;
}

// Simulator::run_with_config's gate loop with a noise model (simulator.rs:67-78):
// every gate, then apply_noise (simulator.rs:177-221) for each qubit of Gate::qubits()
// (gate.rs:40-63; empty for Barrier): depolarising draw (+ the X/Y/Z choice by
// thirds), bit-flip draw, phase-flip draw, each only when its rate is > 0; the
// Paulis go through apply_single_qubit_gate with Gate::matrix_1q.  Draws come from
// the state's stream (the same one measurements use).
int orc_apply_noisy(void* h, const rq_gate* gates, uint64_t n, const double* rates, rq_measurement* out,
                    uint64_t cap, uint64_t* nout) {
    StateBase* s = (StateBase*)h;
    std::vector<rq_measurement> outs;
    const double dep = rates[0], bf = rates[1], pf = rates[2];
    auto pauli = [&](int kind, uint32_t q) {
        rq_gate p{};
        p.kind = kind;
        p.q0 = q;
        M2 m;
        matrix_1q(p, m);
        if (auto d = as<double>(s)) d->apply_1q(q, m); else as<float>(s)->apply_1q(q, m);
    };
    for (uint64_t k = 0; k < n; ++k) {
        const rq_gate& g = gates[k];
        int rc;
        if (auto d = as<double>(s)) rc = apply_gate_impl(d, g, &outs, false);
        else rc = apply_gate_impl(as<float>(s), g, &outs, false);
        if (rc) return rc;
        if (g.kind == RQ_GATE_BARRIER) continue;
        const uint32_t qs[2] = {g.q0, g.q1};
        const int nq = is_2q(g.kind) ? 2 : 1;
        for (int j = 0; j < nq; ++j) {
            const uint32_t q = qs[j];
            if (dep > 0.0) {
                const double r = s->next_uniform();
                if (r < dep) {
                    const double c = s->next_uniform();
                    pauli(c < 1.0 / 3.0 ? RQ_GATE_X : (c < 2.0 / 3.0 ? RQ_GATE_Y : RQ_GATE_Z), q);
                }
            }
            if (bf > 0.0) {
                const double r = s->next_uniform();
                if (r < bf) pauli(RQ_GATE_X, q);
            }
            if (pf > 0.0) {
                const double r = s->next_uniform();
                if (r < pf) pauli(RQ_GATE_Z, q);
            }
        }
    }
    if (nout) *nout = outs.size();
    for (size_t k = 0; k < outs.size() && k < cap; ++k) out[k] = outs[k];
    return RQ_OK;
}

int orc_apply_1q_matrix(void* h, uint32_t q, const double* m8) {
    StateBase* s = (StateBase*)h;
    if (q >= s->nq) return RQ_ERR_INVALID_QUBIT_INDEX;
    M2 m = {{{m8[0], m8[1]}, {m8[2], m8[3]}}, {{m8[4], m8[5]}, {m8[6], m8[7]}}};
    if (auto d = as<double>(s)) d->apply_1q(q, m); else as<float>(s)->apply_1q(q, m);
    return RQ_OK;
}

// One quantum-trajectory step of a single-qubit channel (Kraus operators K_k, row-major 2x2,
// (re, im) pairs).  The reference constructs these sets (noise.rs:166-280) but never applies
// them to a state; this is the standard unravelling the library implements: with
// rho_ij = sum over the pairs differing in bit q of a_i conj(a_j), p_k = tr(K_k rho K_k^+),
// k drawn with the state's next uniform against the normalised cumulative p, and the state
// replaced by K_k psi / sqrt(p_k / sum p).
int orc_apply_kraus(void* h, uint32_t q, const double* kraus, uint32_t nk, int32_t* chosen, double* probability) {
    StateBase* s = (StateBase*)h;
    if (q >= s->nq) return RQ_ERR_INVALID_QUBIT_INDEX;
    if (nk == 0) return RQ_ERR_INVALID_ARGUMENT;
    double r00 = 0, r11 = 0, r01r = 0, r01i = 0;
    auto sums = [&](auto* st) {
        const size_t bit = (size_t)1 << q, n = st->a.size();
        for (size_t i = 0; i < n; ++i) {
            if (i & bit) continue;
            const double a0r = st->a[i].re, a0i = st->a[i].im, a1r = st->a[i | bit].re, a1i = st->a[i | bit].im;
            r00 += a0r * a0r + a0i * a0i;
            r11 += a1r * a1r + a1i * a1i;
            r01r += a0r * a1r + a0i * a1i;   // a0 conj(a1)
            r01i += a0i * a1r - a0r * a1i;
        }
    };
    if (auto d = as<double>(s)) sums(d); else sums(as<float>(s));
    std::vector<double> pk(nk);
    double total = 0;
    for (uint32_t k = 0; k < nk; ++k) {
        const double* K = kraus + 8 * (size_t)k;
        double acc = 0;
        for (int i = 0; i < 2; ++i) {
            const double ar = K[4 * i], ai = K[4 * i + 1], br = K[4 * i + 2], bi = K[4 * i + 3];
            const double cr = ar * r01r - ai * r01i, ci = ar * r01i + ai * r01r;
            acc += (ar * ar + ai * ai) * r00 + (br * br + bi * bi) * r11 + 2.0 * (cr * br + ci * bi);
        }
        pk[k] = acc > 0 ? acc : 0;
        total += pk[k];
    }
    if (!(total > 0)) return RQ_ERR_INVALID_STATE_VECTOR;
    const double u = s->next_uniform();
    uint32_t pick = nk - 1;
    double cum = 0;
    for (uint32_t k = 0; k < nk; ++k) {
        cum += pk[k] / total;
        if (u < cum && pk[k] > 0) { pick = k; break; }
    }
    while (pk[pick] == 0 && pick > 0) --pick;
    const double f = 1.0 / std::sqrt(pk[pick] / total);
    double m8[8];
    for (int j = 0; j < 8; ++j) m8[j] = kraus[8 * (size_t)pick + j] * f;
    orc_apply_1q_matrix(h, q, m8);
    if (chosen) *chosen = (int32_t)pick;
    if (probability) *probability = pk[pick] / total;
    return RQ_OK;
}

int orc_apply_2q_matrix(void* h, uint32_t q1, uint32_t q2, const double* m32) {
    StateBase* s = (StateBase*)h;
    if (q1 >= s->nq || q2 >= s->nq) return RQ_ERR_INVALID_QUBIT_INDEX;
    if (q1 == q2) return RQ_ERR_CIRCUIT;
    M4 m;
    for (int r = 0; r < 4; ++r) for (int c = 0; c < 4; ++c) m[r][c] = {m32[(r * 4 + c) * 2], m32[(r * 4 + c) * 2 + 1]};
    if (auto d = as<double>(s)) d->apply_2q(q1, q2, m); else as<float>(s)->apply_2q(q1, q2, m);
    return RQ_OK;
}

int orc_measure(void* h, uint32_t q, rq_measurement* out) {
    StateBase* s = (StateBase*)h;
    if (q >= s->nq) return RQ_ERR_INVALID_QUBIT_INDEX;
    *out = as<double>(s) ? as<double>(s)->measure(q) : as<float>(s)->measure(q);
    return RQ_OK;
}

int orc_reset_qubit(void* h, uint32_t q) {
    StateBase* s = (StateBase*)h;
    if (q >= s->nq) return RQ_ERR_INVALID_QUBIT_INDEX;
    if (auto d = as<double>(s)) d->reset_qubit(q); else as<float>(s)->reset_qubit(q);
    return RQ_OK;
}

void orc_probabilities(void* h, double* out) {
    auto p = probs_of((StateBase*)h);
    std::memcpy(out, p.data(), p.size() * sizeof(double));
}

double orc_prob_qubit(void* h, uint32_t q) {
    StateBase* s = (StateBase*)h;
    return as<double>(s) ? as<double>(s)->prob_qubit(q) : as<float>(s)->prob_qubit(q);
}

double orc_expectation(void* h, const rq_pauli_op* ops, uint32_t nops) {
    StateBase* s = (StateBase*)h;
    return as<double>(s) ? as<double>(s)->expectation(ops, nops) : as<float>(s)->expectation(ops, nops);
}

// state.rs:403-408: terms summed in order
double orc_expectation_hamiltonian(void* h, const double* coeffs, const rq_pauli_op* ops, const uint32_t* offsets, uint32_t nterms) {
    double acc = 0.0;
    for (uint32_t k = 0; k < nterms; ++k)
        acc += coeffs[k] * orc_expectation(h, ops + offsets[k], offsets[k + 1] - offsets[k]);
    return acc;
}

void orc_normalize(void* h) {
    StateBase* s = (StateBase*)h;
    if (auto d = as<double>(s)) d->normalize(); else as<float>(s)->normalize();
}

// state.rs:426-435
double orc_fidelity(void* ha, void* hb) {
    StateBase* A = (StateBase*)ha; StateBase* B = (StateBase*)hb;
    if (A->nq != B->nq) return 0.0;
    std::vector<double> va((size_t)2 << A->nq), vb((size_t)2 << B->nq);
    auto dl = [](StateBase* s, double* o) {
        if (auto d = as<double>(s)) for (size_t i = 0; i < d->a.size(); ++i) { o[2 * i] = d->a[i].re; o[2 * i + 1] = d->a[i].im; }
        else { auto f = as<float>(s); for (size_t i = 0; i < f->a.size(); ++i) { o[2 * i] = f->a[i].re; o[2 * i + 1] = f->a[i].im; } }
    };
    dl(A, va.data()); dl(B, vb.data());
    C64 inner{0, 0};
    for (size_t i = 0; i < va.size() / 2; ++i)
        inner = cadd(inner, cmul(cconj(C64{va[2 * i], va[2 * i + 1]}), C64{vb[2 * i], vb[2 * i + 1]}));
    return cnorm_sq(inner);
}

void orc_download(void* h, double* out) {
    StateBase* s = (StateBase*)h;
    if (auto d = as<double>(s)) { for (size_t i = 0; i < d->a.size(); ++i) { out[2 * i] = d->a[i].re; out[2 * i + 1] = d->a[i].im; } }
    else { auto f = as<float>(s); for (size_t i = 0; i < f->a.size(); ++i) { out[2 * i] = f->a[i].re; out[2 * i + 1] = f->a[i].im; } }
}

void orc_upload(void* h, const double* in) {
    StateBase* s = (StateBase*)h;
    if (auto d = as<double>(s)) { for (size_t i = 0; i < d->a.size(); ++i) d->a[i] = {in[2 * i], in[2 * i + 1]}; }
    else { auto f = as<float>(s); for (size_t i = 0; i < f->a.size(); ++i) f->a[i] = {(float)in[2 * i], (float)in[2 * i + 1]}; }
}

uint64_t orc_draws(void* h) { return ((StateBase*)h)->draws; }

// Simulator::run_shots, literally (simulator.rs:107-147): re-simulate the
// whole circuit per shot with seed base+shot, then measure_all when the
// circuit has no Measure gate.  bits[s]: bit q = last outcome of qubit q.
int orc_run_shots_literal(uint32_t nq, int32_t prec, const rq_gate* gates, uint64_t ngates,
                          uint64_t shots, uint64_t base_seed, uint64_t* out_bits) {
    bool has_meas = false;
    for (uint64_t k = 0; k < ngates; ++k) has_meas |= gates[k].kind == RQ_GATE_MEASURE;
    for (uint64_t s = 0; s < shots; ++s) {
        void* h = nullptr;
        int rc = orc_state_new(nq, prec, base_seed + s, 1, &h);
        if (rc) return rc;
        std::vector<rq_measurement> outs(ngates + nq + 1);
        uint64_t nout = 0;
        rc = orc_apply(h, gates, ngates, outs.data(), outs.size(), &nout, 0);
        if (rc) { orc_state_free(h); return rc; }
        outs.resize(nout);
        if (!has_meas) {
            for (uint32_t q = 0; q < nq; ++q) { rq_measurement m; orc_measure(h, q, &m); outs.push_back(m); }
        }
        uint64_t bits = 0;
        for (auto& m : outs) {
            if (m.result) bits |= (uint64_t)1 << m.qubit; else bits &= ~((uint64_t)1 << m.qubit);
        }
        out_bits[s] = bits;
        orc_state_free(h);
    }
    return RQ_OK;
}

void orc_tree_sample(const double* probs, uint32_t n, const uint32_t* qubits, uint32_t m,
                     uint64_t base_seed, uint64_t shots, uint64_t* out_bits) {
    tree_sample(probs, n, qubits, m, base_seed, shots, out_bits);
}

// ---------------------------------------------------------------------------
// ruqu-algorithms drivers, restated (qaoa.rs:125-308, vqe.rs:65-216)
// ---------------------------------------------------------------------------

// build_qaoa_circuit (qaoa.rs:125-153)
static std::vector<rq_gate> qaoa_circuit(uint32_t n, const uint32_t* ei, const uint32_t* ej, const double* w, uint32_t ne,
                                         const double* gammas, const double* betas, uint32_t p) {
    std::vector<rq_gate> c;
    for (uint32_t q = 0; q < n; ++q) { rq_gate g{}; g.kind = RQ_GATE_H; g.q0 = q; c.push_back(g); }
    for (uint32_t l = 0; l < p; ++l) {
        for (uint32_t e = 0; e < ne; ++e) { rq_gate g{}; g.kind = RQ_GATE_RZZ; g.q0 = ei[e]; g.q1 = ej[e]; g.angle = 2.0 * gammas[l] * w[e]; c.push_back(g); }
        for (uint32_t q = 0; q < n; ++q) { rq_gate g{}; g.kind = RQ_GATE_RX; g.q0 = q; g.angle = 2.0 * betas[l]; c.push_back(g); }
    }
    return c;
}

// evaluate_qaoa_cost (qaoa.rs:179-201); prec selects the f64 or f32 engine
double orc_qaoa_cost(uint32_t n, const uint32_t* ei, const uint32_t* ej, const double* w, uint32_t ne,
                     const double* gammas, const double* betas, uint32_t p, int32_t prec) {
    auto c = qaoa_circuit(n, ei, ej, w, ne, gammas, betas, p);
    void* h = nullptr;
    if (orc_state_new(n, prec, 0, 1, &h)) return NAN;
    orc_apply(h, c.data(), c.size(), nullptr, 0, nullptr, 0);
    double cost = 0.0;
    for (uint32_t e = 0; e < ne; ++e) {
        rq_pauli_op ops[2] = {{ei[e], RQ_PAULI_Z}, {ej[e], RQ_PAULI_Z}};
        double zz = orc_expectation(h, ops, 2);
        cost += w[e] * 0.5 * (1.0 - zz);
    }
    orc_state_free(h);
    return cost;
}

// Final-state probabilities of the QAOA circuit (for best-bitstring checks).
void orc_qaoa_probabilities(uint32_t n, const uint32_t* ei, const uint32_t* ej, const double* w, uint32_t ne,
                            const double* gammas, const double* betas, uint32_t p, int32_t prec, double* out) {
    auto c = qaoa_circuit(n, ei, ej, w, ne, gammas, betas, p);
    void* h = nullptr;
    orc_state_new(n, prec, 0, 1, &h);
    orc_apply(h, c.data(), c.size(), nullptr, 0, nullptr, 0);
    orc_probabilities(h, out);
    orc_state_free(h);
}

// run_qaoa (qaoa.rs:217-308): gradient ascent with the parameter-shift rule
// from gamma = beta = 0.5; best bitstring = argmax of the final probabilities
// whenever the cost improves (first maximum wins, as Iterator::max_by keeps
// the last of equal elements -- see the comparator note below).
int orc_run_qaoa(uint32_t n, const uint32_t* ei, const uint32_t* ej, const double* w, uint32_t ne,
                 uint32_t p, uint32_t max_iter, double lr,
                 double* out_gammas, double* out_betas, double* out_history, uint32_t* out_iters,
                 double* out_best_cost, uint64_t* out_best_bits, int32_t* out_converged) {
    std::vector<double> g(p, 0.5), b(p, 0.5);
    std::vector<double> hist;
    double best = -INFINITY;
    uint64_t best_bits = 0;
    int converged = 0;
    const double shift = 1.57079632679489661923;
    for (uint32_t it = 0; it < max_iter; ++it) {
        double cost = orc_qaoa_cost(n, ei, ej, w, ne, g.data(), b.data(), p, RQ_F64);
        hist.push_back(cost);
        if (cost > best) {
            best = cost;
            std::vector<double> pr((size_t)1 << n);
            orc_qaoa_probabilities(n, ei, ej, w, ne, g.data(), b.data(), p, RQ_F64, pr.data());
            // Iterator::max_by returns the LAST maximal element on ties.
            size_t bi = 0;
            for (size_t i = 1; i < pr.size(); ++i) if (!(pr[i] < pr[bi])) bi = i;
            best_bits = bi;
        }
        if (it > 0 && std::fabs(cost - hist[it - 1]) < 1e-6) { converged = 1; break; }
        for (uint32_t i = 0; i < p; ++i) {
            std::vector<double> gp = g, gm = g; gp[i] += shift; gm[i] -= shift;
            double cp = orc_qaoa_cost(n, ei, ej, w, ne, gp.data(), b.data(), p, RQ_F64);
            double cm = orc_qaoa_cost(n, ei, ej, w, ne, gm.data(), b.data(), p, RQ_F64);
            g[i] += lr * (cp - cm) / 2.0;
        }
        for (uint32_t i = 0; i < p; ++i) {
            std::vector<double> bp = b, bm = b; bp[i] += shift; bm[i] -= shift;
            double cp = orc_qaoa_cost(n, ei, ej, w, ne, g.data(), bp.data(), p, RQ_F64);
            double cm = orc_qaoa_cost(n, ei, ej, w, ne, g.data(), bm.data(), p, RQ_F64);
            b[i] += lr * (cp - cm) / 2.0;
        }
    }
    std::copy(g.begin(), g.end(), out_gammas);
    std::copy(b.begin(), b.end(), out_betas);
    std::copy(hist.begin(), hist.end(), out_history);
    *out_iters = (uint32_t)hist.size();
    *out_best_cost = best;
    *out_best_bits = best_bits;
    *out_converged = converged;
    return RQ_OK;
}

// Energy of an arbitrary gate list under a Hamiltonian (evaluate_energy,
// vqe.rs:122-131, with the ansatz supplied as a gate list).
double orc_circuit_energy(uint32_t n, int32_t prec, const rq_gate* gates, uint64_t ngates,
                          const double* coeffs, const rq_pauli_op* ops, const uint32_t* offsets, uint32_t nterms) {
    void* h = nullptr;
    if (orc_state_new(n, prec, 0, 1, &h)) return NAN;
    orc_apply(h, gates, ngates, nullptr, 0, nullptr, 0);
    double e = orc_expectation_hamiltonian(h, coeffs, ops, offsets, nterms);
    orc_state_free(h);
    return e;
}

// build_ansatz (vqe.rs:81-112): per layer Ry on all, Rz on all, CNOT chain
static std::vector<rq_gate> vqe_ansatz(uint32_t n, uint32_t depth, const double* params) {
    std::vector<rq_gate> c;
    size_t idx = 0;
    for (uint32_t l = 0; l < depth; ++l) {
        for (uint32_t q = 0; q < n; ++q) { rq_gate g{}; g.kind = RQ_GATE_RY; g.q0 = q; g.angle = params[idx++]; c.push_back(g); }
        for (uint32_t q = 0; q < n; ++q) { rq_gate g{}; g.kind = RQ_GATE_RZ; g.q0 = q; g.angle = params[idx++]; c.push_back(g); }
        for (uint32_t q = 0; q + 1 < n; ++q) { rq_gate g{}; g.kind = RQ_GATE_CNOT; g.q0 = q; g.q1 = q + 1; c.push_back(g); }
    }
    return c;
}

// run_vqe (vqe.rs:148-216): params start at 0.1, parameter-shift gradient
// descent, best energy tracked, convergence on |dE| < threshold.
int orc_run_vqe(uint32_t n, uint32_t depth, const double* coeffs, const rq_pauli_op* ops, const uint32_t* offsets,
                uint32_t nterms, uint32_t max_iter, double threshold, double lr,
                double* out_best_params, double* out_history, uint32_t* out_iters, double* out_best_energy,
                int32_t* out_converged) {
    size_t np = 2ull * n * depth;
    std::vector<double> params(np, 0.1), best_params = params;
    std::vector<double> hist;
    double best = 1.7976931348623157e308;
    int converged = 0;
    const double shift = 1.57079632679489661923;
    auto energy = [&](const std::vector<double>& pr) {
        auto c = vqe_ansatz(n, depth, pr.data());
        return orc_circuit_energy(n, RQ_F64, c.data(), c.size(), coeffs, ops, offsets, nterms);
    };
    for (uint32_t it = 0; it < max_iter; ++it) {
        double e = energy(params);
        hist.push_back(e);
        if (e < best) { best = e; best_params = params; }
        if (it > 0 && std::fabs(hist[it - 1] - e) < threshold) { converged = 1; break; }
        std::vector<double> grad(np);
        for (size_t i = 0; i < np; ++i) {
            std::vector<double> pp = params, pm = params;
            pp[i] += shift; pm[i] -= shift;
            grad[i] = (energy(pp) - energy(pm)) / 2.0;
        }
        for (size_t i = 0; i < np; ++i) params[i] -= lr * grad[i];
    }
    std::copy(best_params.begin(), best_params.end(), out_best_params);
    std::copy(hist.begin(), hist.end(), out_history);
    *out_iters = (uint32_t)hist.size();
    *out_best_energy = best;
    *out_converged = converged;
    return RQ_OK;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
