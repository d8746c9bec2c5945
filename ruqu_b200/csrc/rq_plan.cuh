// rq_plan.cuh -- host planner of multi-gate sweeps, shared by the single-state
// sweep path (rq_sweep.cu) and the batched QAOA / VQE engines (rq_batch.cu).
//
// A sweep owns m local qubits (qubits 0..c-1 always among them) and runs in
// phases; in a phase every thread holds 2^RB amplitudes whose indices differ
// in RB register slots.  The planner keeps per-qubit gate order: it scans the
// remaining gates and takes every gate none of whose qubits is held back by an
// earlier untaken gate (gates on disjoint qubits commute).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <utility>
#include <vector>

#include "rq_internal.cuh"

namespace rqp {

// Device op kinds.  U1: dense 2x2 from the matrix table; D1: diagonal 2x2;
// CX/CZ/ZZ: CNOT, CZ, Rzz-type diagonal; CPH: MaxCut cost phase
// exp(-i*gamma_l*(|E| - 2 cut(x))) over all qubits (param = layer l);
// RXP / RYP: Rx / Ry whose angle comes from the circuit's parameter table
// (param = its index there).
// DENSE: a 32x32 complex unitary on the phase's five register slots, applied
// on the tensor cores (param = index of its operand image).
enum OpType : uint8_t { OP_U1 = 0, OP_D1 = 1, OP_CX = 2, OP_CZ = 3, OP_ZZ = 4, OP_CPH = 5, OP_RXP = 6, OP_RYP = 7,
                        OP_DENSE = 8 };

constexpr int RBMAX = 5;
constexpr int MMAX = 14;

struct __align__(16) SwOp {
    uint8_t type;
    int8_t k0, k1;   // register slot of q0 / q1 in this phase, -1 if not a slot
    uint8_t q0, q1;  // global qubits
    uint8_t pad;
    uint16_t param;  // layer / parameter index of CPH, RXP, RYP
    uint32_t mat;    // first complex entry in the matrix table
    uint32_t pad2;
};

struct __align__(16) PhaseDesc {
    uint32_t slut[1 << RBMAX];   // swz(lut[i]) for the state's element size
    uint16_t tsw[8];             // FP16 tensor-core plans: swz16 of thread bit b's local offset
    uint32_t op_begin, op_end;
    uint32_t nt;                 // number of thread bits
    uint8_t tbit_local[12];      // thread bit b -> local bit index (nt <= MMAX - 4)
    uint8_t tbit_global[12];     // thread bit b -> global qubit
    uint16_t lut[1 << RBMAX];    // register index -> local offset
    uint8_t slot_global[RBMAX];  // register slot -> global qubit
};
static_assert(sizeof(PhaseDesc) == 256, "phase descriptors are copied in 16-byte units");

struct SweepDesc {
    uint32_t n, m, c;
    uint32_t nonlocal_count;
    uint8_t local_global[32];   // local bit -> global qubit
    uint8_t nonlocal[64];       // non-local bits in ascending order
    uint32_t phase_begin, phase_end;
    uint32_t flags;             // SWEEP_INIT_UNIFORM | SWEEP_ENERGY (batched sweeps)
    uint64_t gj[1 << RBMAX];    // deposit of the per-thread vector offsets
    uint32_t sgj[1 << RBMAX];   // swz((tid-independent part of) the vector's first element)
    uint32_t img_begin, img_count;   // dense operand images of this sweep (tensor-core sweeps)
};

constexpr uint32_t SWEEP_INIT_UNIFORM = 1u;   // synthesise |+>^n instead of loading the tile
constexpr uint32_t SWEEP_ENERGY = 2u;         // reduce sum |a|^2 cut(x) after the last phase
constexpr uint32_t SWEEP_INIT_ZERO = 4u;      // synthesise |0...0> instead of loading the tile
constexpr uint32_t SWEEP_INIT_LAMBDA = 8u;    // adjoint sweeps: build lambda = C psi instead of loading it
// batched QAOA: Rx(t) = S^dag Ry(t) S, and the S of one layer cancels the S^dag of the next
// across the diagonal cost phase, so the forward program runs Ry and carries the phases
// i^popc(x) from the start (PHASE_IN, with INIT_UNIFORM) to the end (PHASE_OUT: (-i)^popc(x)
// after the last phase)
constexpr uint32_t SWEEP_PHASE_IN = 16u;
constexpr uint32_t SWEEP_PHASE_OUT = 32u;


struct PGate {
    uint8_t type;
    uint32_t q0, q1;
    double m[8];          // U1: 2x2; D1: d0,d1; ZZ: en,ep
    uint16_t param = 0;   // CPH / RXP / RYP
    uint64_t span = 0;    // qubits touched when not just q0/q1 (CPH: all)
};

inline uint64_t qmask(const PGate& g) {
    if (g.span) return g.span;
    uint64_t m = 1ull << g.q0;
    if (g.type == OP_CX || g.type == OP_CZ || g.type == OP_ZZ) m |= 1ull << g.q1;
    return m;
}

// qubits that must be register slots (and therefore local).  With all_slots
// (plans for dense tensor-core phases) every qubit a 1- or 2-qubit gate touches
// is a slot, so whole gate runs stay inside the phase's 32-dimensional space.
inline uint64_t needs(const PGate& g, bool all_slots = false) {
    if (g.type == OP_U1 || g.type == OP_RXP || g.type == OP_RYP) return 1ull << g.q0;
    if (all_slots) {
        if (g.type == OP_D1) return 1ull << g.q0;
        if (g.type == OP_CX || g.type == OP_CZ || g.type == OP_ZZ) return (1ull << g.q0) | (1ull << g.q1);
    }
    if (g.type == OP_CX) return 1ull << g.q1;
    return 0;
}

// 1-qubit gates whose matrices the planner may multiply together
inline bool is_1q(uint8_t t) { return t == OP_U1 || t == OP_D1; }

// c = a * b (2x2 complex, row-major (re,im))
inline void mat2_mul(const double* a, const double* b, double* c) {
    double r[8];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) {
            double re = 0, im = 0;
            for (int k = 0; k < 2; ++k) {
                double ar = a[(i * 2 + k) * 2], ai = a[(i * 2 + k) * 2 + 1];
                double br = b[(k * 2 + j) * 2], bi = b[(k * 2 + j) * 2 + 1];
                re += ar * br - ai * bi;
                im += ar * bi + ai * br;
            }
            r[(i * 2 + j) * 2] = re;
            r[(i * 2 + j) * 2 + 1] = im;
        }
    std::memcpy(c, r, sizeof(r));
}

inline void as_matrix(const PGate& g, double* m) {
    if (g.type == OP_U1) {
        std::memcpy(m, g.m, sizeof(double) * 8);
    } else {  // D1
        double r[8] = {g.m[0], g.m[1], 0, 0, 0, 0, g.m[2], g.m[3]};
        std::memcpy(m, r, sizeof(r));
    }
}

// fuse `nxt` (applied after `cur`) into cur; both 1-qubit on the same qubit
inline void fuse_into(PGate& cur, const PGate& nxt) {
    if (cur.type == OP_D1 && nxt.type == OP_D1) {
        double a[2] = {cur.m[0], cur.m[1]}, b[2] = {cur.m[2], cur.m[3]};
        cur.m[0] = nxt.m[0] * a[0] - nxt.m[1] * a[1];
        cur.m[1] = nxt.m[0] * a[1] + nxt.m[1] * a[0];
        cur.m[2] = nxt.m[2] * b[0] - nxt.m[3] * b[1];
        cur.m[3] = nxt.m[2] * b[1] + nxt.m[3] * b[0];
        return;
    }
    double A[8], B[8], C[8];
    as_matrix(cur, A);
    as_matrix(nxt, B);
    mat2_mul(B, A, C);
    cur.type = OP_U1;
    std::memcpy(cur.m, C, sizeof(C));
}

struct Sweep {
    uint64_t L;               // local qubit mask
    std::vector<PGate> ops;   // in execution order (after fusion)
};

// First-come local sets: each sweep admits the qubits of the remaining gates in list
// order until m are local.
inline std::vector<Sweep> plan_sweeps_first_come(const std::vector<PGate>& gates, uint32_t n, uint32_t m,
                                                 uint32_t c) {
    std::vector<Sweep> out;
    std::vector<char> taken(gates.size(), 0);
    size_t first = 0;
    const uint64_t base = (c >= 64) ? ~0ull : ((1ull << c) - 1);
    while (first < gates.size()) {
        Sweep sw;
        sw.L = base;
        uint64_t blocked = 0;
        std::vector<int> last(n, -1);   // index in sw.ops of the last op on each qubit
        for (size_t k = first; k < gates.size(); ++k) {
            if (taken[k]) continue;
            const PGate& g = gates[k];
            uint64_t qm = qmask(g);
            if (qm & blocked) {
                blocked |= qm;
                continue;
            }
            uint64_t L2 = sw.L | needs(g, false);
            if ((uint32_t)__builtin_popcountll(L2) > m) {
                blocked |= qm;
                continue;
            }
            sw.L = L2;
            taken[k] = 1;
            if (is_1q(g.type) && last[g.q0] >= 0 && is_1q(sw.ops[last[g.q0]].type)) {
                fuse_into(sw.ops[last[g.q0]], g);
            } else {
                sw.ops.push_back(g);
                int idx = (int)sw.ops.size() - 1;
                for (uint32_t q = 0; q < n; ++q)
                    if ((qm >> q) & 1) last[q] = idx;
            }
        }
        while (first < gates.size() && taken[first]) ++first;
        out.push_back(std::move(sw));
    }
    return out;
}

// Gates a sweep with the fixed local set L would take from the remaining list (per-qubit
// order kept: a gate that cannot run holds its qubits back for the rest of the list);
// marks them in *mark when given.  Stops once every qubit is held back.
inline int sweep_closure(const std::vector<PGate>& gates, const std::vector<char>& taken, size_t first, uint64_t L,
                         uint64_t allq, std::vector<char>* mark) {
    uint64_t blocked = 0;
    int cnt = 0;
    for (size_t k = first; k < gates.size(); ++k) {
        if (taken[k]) continue;
        const PGate& g = gates[k];
        const uint64_t qm = qmask(g);
        if ((qm & blocked) || (needs(g, false) & ~L)) {
            blocked |= qm;
            if ((blocked & allq) == allq) break;
            continue;
        }
        ++cnt;
        if (mark) (*mark)[k] = 1;
    }
    return cnt;
}

// Candidate local sets for the next sweep: the first-come set (padded to m qubits) and
// every window of m - c consecutive qubits above the always-local low c qubits (the
// shape that follows nearest-neighbour circuits as their light cones move).
inline std::vector<uint64_t> sweep_candidates(const std::vector<PGate>& gates, const std::vector<char>& taken,
                                              size_t first, uint32_t n, uint32_t m, uint32_t c) {
    const uint64_t base = (c >= 64) ? ~0ull : ((1ull << c) - 1);
    std::vector<uint64_t> out;
    uint64_t L = base, blocked = 0;
    for (size_t k = first; k < gates.size(); ++k) {
        if (taken[k]) continue;
        const uint64_t qm = qmask(gates[k]);
        if (qm & blocked) { blocked |= qm; continue; }
        const uint64_t L2 = L | needs(gates[k], false);
        if ((uint32_t)__builtin_popcountll(L2) > m) { blocked |= qm; continue; }
        L = L2;
    }
    for (uint32_t q = 0; q < n && (uint32_t)__builtin_popcountll(L) < m; ++q) L |= 1ull << q;
    out.push_back(L);
    const uint32_t w = m > c ? m - c : 0;
    for (uint32_t a0 = c; w && a0 + w <= n; ++a0) {
        uint64_t W = base;
        for (uint32_t q = a0; q < a0 + w; ++q) W |= 1ull << q;
        if (W != L) out.push_back(W);
    }
    return out;
}

// Lookahead local sets: each sweep takes the candidate set that maximises the gates it
// runs plus the most the following sweep could then run (two-step lookahead over the
// candidates of sweep_candidates).
inline std::vector<Sweep> plan_sweeps_lookahead(const std::vector<PGate>& gates, uint32_t n, uint32_t m, uint32_t c) {
    std::vector<Sweep> out;
    std::vector<char> taken(gates.size(), 0);
    const uint64_t allq = (n >= 64) ? ~0ull : ((1ull << n) - 1);
    size_t first = 0;
    while (first < gates.size()) {
        const auto cands = sweep_candidates(gates, taken, first, n, m, c);
        double best = -1.0;
        uint64_t bestL = cands[0];
        for (uint64_t L : cands) {
            std::vector<char> t2 = taken;
            double score = sweep_closure(gates, taken, first, L, allq, &t2);
            size_t f2 = first;
            while (f2 < gates.size() && t2[f2]) ++f2;
            int next = 0;
            if (f2 < gates.size())
                for (uint64_t L2 : sweep_candidates(gates, t2, f2, n, m, c))
                    next = std::max(next, sweep_closure(gates, t2, f2, L2, allq, nullptr));
            score += 0.999 * next;   // ties go to the set that runs more gates now
            if (score > best) {
                best = score;
                bestL = L;
            }
        }
        Sweep sw;
        sw.L = bestL;
        std::vector<int> last(n, -1);   // index in sw.ops of the last op on each qubit
        uint64_t blocked = 0;
        for (size_t k = first; k < gates.size(); ++k) {
            if (taken[k]) continue;
            const PGate& g = gates[k];
            const uint64_t qm = qmask(g);
            if ((qm & blocked) || (needs(g, false) & ~bestL)) {
                blocked |= qm;
                continue;
            }
            taken[k] = 1;
            if (is_1q(g.type) && last[g.q0] >= 0 && is_1q(sw.ops[last[g.q0]].type)) {
                fuse_into(sw.ops[last[g.q0]], g);
            } else {
                sw.ops.push_back(g);
                const int idx = (int)sw.ops.size() - 1;
                for (uint32_t q = 0; q < n; ++q)
                    if ((qm >> q) & 1) last[q] = idx;
            }
        }
        while (first < gates.size() && taken[first]) ++first;
        out.push_back(std::move(sw));
    }
    return out;
}

constexpr int DENSE_MAX_VQ_PLAN = 4;   // qubits outside the tile per tensor-core phase (2^4 image variants)

struct PhasePlan {
    uint64_t R;               // register qubits (global mask)
    std::vector<int> ops;     // indices into the sweep's op list
};

// First-come register slots: each phase admits the slot qubits of the sweep's remaining
// ops in order until rb are taken.
inline std::vector<PhasePlan> plan_phases_first_come(const Sweep& sw, uint32_t rb, bool all_slots) {
    std::vector<PhasePlan> out;
    std::vector<char> taken(sw.ops.size(), 0);
    size_t first = 0;
    while (first < sw.ops.size()) {
        PhasePlan ph;
        ph.R = 0;
        uint64_t blocked = 0;
        uint64_t outside = 0;   // tensor-core plans: gate qubits outside the tile used by the phase
        for (size_t k = first; k < sw.ops.size(); ++k) {
            if (taken[k]) continue;
            const PGate& g = sw.ops[k];
            uint64_t qm = qmask(g);
            if (qm & blocked) {
                blocked |= qm;
                continue;
            }
            // tensor-core plans: every local qubit of the gate is a register slot, and the phase
            // uses at most DENSE_MAX_VQ qubits outside the tile (one operand image per assignment)
            uint64_t R2 = ph.R | needs(g, false) | (all_slots ? (qm & sw.L) : 0ull);
            const uint64_t out2 = all_slots ? (outside | (qm & ~sw.L)) : 0ull;
            if ((uint32_t)__builtin_popcountll(R2) > rb || __builtin_popcountll(out2) > DENSE_MAX_VQ_PLAN) {
                blocked |= qm;
                continue;
            }
            outside = out2;
            ph.R = R2;
            taken[k] = 1;
            ph.ops.push_back((int)k);
        }
        // fill the remaining slots with the lowest unused local qubits
        for (uint32_t q = 0; q < 64 && (uint32_t)__builtin_popcountll(ph.R) < rb; ++q)
            if (((sw.L >> q) & 1) && !((ph.R >> q) & 1)) ph.R |= 1ull << q;
        while (first < sw.ops.size() && taken[first]) ++first;
        out.push_back(std::move(ph));
    }
    return out;
}

// Ops of the sweep a phase with slot set R would take (per-qubit order kept), with the
// same rules as plan_phases_first_come; marks them in *mark when given.
inline int phase_closure(const Sweep& sw, const std::vector<char>& taken, size_t first, uint64_t R, bool all_slots,
                         std::vector<int>* mark) {
    uint64_t blocked = 0, outside = 0;
    int cnt = 0;
    for (size_t k = first; k < sw.ops.size(); ++k) {
        if (taken[k]) continue;
        const PGate& g = sw.ops[k];
        const uint64_t qm = qmask(g);
        const uint64_t need = needs(g, false) | (all_slots ? (qm & sw.L) : 0ull);
        const uint64_t out2 = all_slots ? (outside | (qm & ~sw.L)) : 0ull;
        if ((qm & blocked) || (need & ~R) || __builtin_popcountll(out2) > DENSE_MAX_VQ_PLAN) {
            blocked |= qm;
            continue;
        }
        outside = out2;
        ++cnt;
        if (mark) mark->push_back((int)k);
    }
    return cnt;
}

// Lookahead register slots: candidates are the first-come slot set and every window of
// rb consecutive local qubits; each phase takes the one maximising the ops it runs plus
// the most the next phase could then run.
inline std::vector<PhasePlan> plan_phases_lookahead(const Sweep& sw, uint32_t rb, bool all_slots) {
    std::vector<PhasePlan> out;
    std::vector<char> taken(sw.ops.size(), 0);
    std::vector<uint32_t> loc;
    for (uint32_t q = 0; q < 64; ++q)
        if ((sw.L >> q) & 1) loc.push_back(q);
    auto cands = [&](const std::vector<char>& tk, size_t f) {
        std::vector<uint64_t> c;
        // the first-come choice for the remaining ops
        uint64_t R = 0, blocked = 0, outside = 0;
        for (size_t k = f; k < sw.ops.size(); ++k) {
            if (tk[k]) continue;
            const PGate& g = sw.ops[k];
            const uint64_t qm = qmask(g);
            if (qm & blocked) { blocked |= qm; continue; }
            const uint64_t R2 = R | needs(g, false) | (all_slots ? (qm & sw.L) : 0ull);
            const uint64_t out2 = all_slots ? (outside | (qm & ~sw.L)) : 0ull;
            if ((uint32_t)__builtin_popcountll(R2) > rb || __builtin_popcountll(out2) > DENSE_MAX_VQ_PLAN) {
                blocked |= qm;
                continue;
            }
            R = R2;
            outside = out2;
        }
        for (uint32_t q : loc)
            if ((uint32_t)__builtin_popcountll(R) < rb && !((R >> q) & 1)) R |= 1ull << q;
        c.push_back(R);
        for (size_t a0 = 0; a0 + rb <= loc.size(); ++a0) {
            uint64_t W = 0;
            for (size_t j = a0; j < a0 + rb; ++j) W |= 1ull << loc[j];
            if (W != R) c.push_back(W);
        }
        return c;
    };
    size_t first = 0;
    while (first < sw.ops.size()) {
        const auto c = cands(taken, first);
        double best = -1.0;
        uint64_t bestR = c[0];
        for (uint64_t R : c) {
            std::vector<int> got;
            double score = phase_closure(sw, taken, first, R, all_slots, &got);
            if (got.empty()) continue;
            std::vector<char> t2 = taken;
            for (int k : got) t2[k] = 1;
            size_t f2 = first;
            while (f2 < sw.ops.size() && t2[f2]) ++f2;
            int next = 0;
            if (f2 < sw.ops.size())
                for (uint64_t R2 : cands(t2, f2)) next = std::max(next, phase_closure(sw, t2, f2, R2, all_slots, nullptr));
            score += 0.999 * next;   // ties go to the set that runs more ops now
            if (score > best) {
                best = score;
                bestR = R;
            }
        }
        PhasePlan ph;
        ph.R = bestR;
        if (phase_closure(sw, taken, first, bestR, all_slots, &ph.ops) == 0) return {};   // no progress: give up
        for (int k : ph.ops) taken[k] = 1;
        while (first < sw.ops.size() && taken[first]) ++first;
        out.push_back(std::move(ph));
    }
    return out;
}

// Beam search over phase plans: breadth-first by phase, each partial plan extended by every
// slot set of the lookahead planner's candidates (the first-come set for its remaining ops,
// every window of rb consecutive local qubits); of the extensions, the `width` that have run
// the most ops (distinct sets of ops) are kept.  The first partial plan that runs every op
// is returned, so no plan the beam saw has fewer phases.  Empty when no extension makes
// progress.
inline std::vector<PhasePlan> plan_phases_beam(const Sweep& sw, uint32_t rb, bool all_slots, size_t width = 8) {
    struct Partial {
        std::vector<char> taken;
        size_t first;
        int done;
        std::vector<PhasePlan> phases;
    };
    std::vector<uint32_t> loc;
    for (uint32_t q = 0; q < 64; ++q)
        if ((sw.L >> q) & 1) loc.push_back(q);
    auto cands = [&](const std::vector<char>& tk, size_t f) {
        std::vector<uint64_t> c;
        uint64_t R = 0, blocked = 0, outside = 0;
        for (size_t k = f; k < sw.ops.size(); ++k) {
            if (tk[k]) continue;
            const PGate& g = sw.ops[k];
            const uint64_t qm = qmask(g);
            if (qm & blocked) { blocked |= qm; continue; }
            const uint64_t R2 = R | needs(g, false) | (all_slots ? (qm & sw.L) : 0ull);
            const uint64_t out2 = all_slots ? (outside | (qm & ~sw.L)) : 0ull;
            if ((uint32_t)__builtin_popcountll(R2) > rb || __builtin_popcountll(out2) > DENSE_MAX_VQ_PLAN) {
                blocked |= qm;
                continue;
            }
            R = R2;
            outside = out2;
        }
        for (uint32_t q : loc)
            if ((uint32_t)__builtin_popcountll(R) < rb && !((R >> q) & 1)) R |= 1ull << q;
        c.push_back(R);
        for (size_t a0 = 0; a0 + rb <= loc.size(); ++a0) {
            uint64_t W = 0;
            for (size_t j = a0; j < a0 + rb; ++j) W |= 1ull << loc[j];
            if (W != R) c.push_back(W);
        }
        return c;
    };
    if (sw.ops.empty()) return {};
    std::vector<Partial> beam(1);
    beam[0].taken.assign(sw.ops.size(), 0);
    beam[0].first = 0;
    beam[0].done = 0;
    for (size_t depth = 1; depth <= sw.ops.size(); ++depth) {
        std::vector<Partial> next;
        std::vector<std::vector<char>> seen;
        for (const Partial& p : beam)
            for (uint64_t R : cands(p.taken, p.first)) {
                PhasePlan ph;
                ph.R = R;
                if (phase_closure(sw, p.taken, p.first, R, all_slots, &ph.ops) == 0) continue;
                Partial t{p.taken, p.first, p.done + (int)ph.ops.size(), p.phases};
                for (int k : ph.ops) t.taken[k] = 1;
                while (t.first < sw.ops.size() && t.taken[t.first]) ++t.first;
                t.phases.push_back(std::move(ph));
                if (t.first >= sw.ops.size()) return t.phases;
                if (std::find(seen.begin(), seen.end(), t.taken) != seen.end()) continue;
                seen.push_back(t.taken);
                next.push_back(std::move(t));
            }
        std::stable_sort(next.begin(), next.end(), [](const Partial& a, const Partial& b) { return a.done > b.done; });
        if (next.size() > width) next.resize(width);
        if (next.empty()) return {};
        beam = std::move(next);
    }
    return {};
}

// The phase plan: the first-come and lookahead planners, keeping the one with fewer phases
// (first-come on a tie or when the lookahead finds no progress); tensor-core plans
// (all_slots, where a phase is a dense MMA round trip) also run the beam search and take its
// plan when it has fewer phases still (the 30-qubit random-layer circuit: 52 -> 50 phases
// over the same 14 sweeps of 13 local qubits).
inline std::vector<PhasePlan> plan_phases(const Sweep& sw, uint32_t rb, bool all_slots = false) {
    auto a = plan_phases_first_come(sw, rb, all_slots);
    auto b = plan_phases_lookahead(sw, rb, all_slots);
    auto best = (!b.empty() && b.size() < a.size()) ? b : a;
    if (!all_slots) return best;
    auto c = plan_phases_beam(sw, rb, all_slots);
    return (!c.empty() && c.size() < best.size()) ? c : best;
}

// Gates the fixed local set L takes, as a sweep (1-qubit runs fused), marking them taken.
inline Sweep take_sweep(const std::vector<PGate>& gates, std::vector<char>& taken, size_t first, uint64_t L,
                        uint32_t n, uint32_t m) {
    Sweep sw;
    sw.L = L;
    std::vector<int> last(n, -1);
    uint64_t blocked = 0;
    for (size_t k = first; k < gates.size(); ++k) {
        if (taken[k]) continue;
        const PGate& g = gates[k];
        const uint64_t qm = qmask(g);
        if ((qm & blocked) || (needs(g, false) & ~L)) {
            blocked |= qm;
            continue;
        }
        taken[k] = 1;
        if (is_1q(g.type) && last[g.q0] >= 0 && is_1q(sw.ops[last[g.q0]].type)) {
            fuse_into(sw.ops[last[g.q0]], g);
        } else {
            sw.ops.push_back(g);
            const int idx = (int)sw.ops.size() - 1;
            for (uint32_t q = 0; q < n; ++q)
                if ((qm >> q) & 1) last[q] = idx;
        }
    }
    for (uint32_t q = 0; q < n && (uint32_t)__builtin_popcountll(sw.L) < m; ++q) sw.L |= 1ull << q;
    return sw;
}

// Tensor-core sweep cost model: a launch costs about sweep + phase x its phases.  Least-
// squares fits of the per-launch times of the 30-qubit f32 benchmark circuit (launch lists
// of one step; both terms scale with the state size, so only their ratio matters here):
//   3xTF32 sweeps (two MMA round trips per phase): 1.79 ms + 1.91 ms per phase;
//   FP16-split sweeps (one round trip):             3.15 ms + 1.05 ms per phase.
struct SweepCost {
    double sweep, phase;
};
constexpr SweepCost COST_TF32{1.79, 1.91}, COST_F16{3.15, 1.05};

// The autotuner's choice among timed candidates: candidate 0 is the reference point, and a
// later eligible candidate replaces the best so far only when it is faster by more than the
// relative margin, so near-equal plans keep the earlier one (the candidates are listed with
// fewer sweeps first) instead of following timing noise.
inline size_t pick_fastest(const float* ms, const bool* eligible, size_t n, float margin = 0.02f) {
    size_t best = 0;
    for (size_t k = 1; k < n; ++k)
        if (eligible[k] && ms[k] < (1.f - margin) * ms[best]) best = k;
    return best;
}

inline double plan_cost(std::vector<Sweep> sweeps, uint32_t n, uint32_t m, uint32_t rb, SweepCost k = COST_TF32) {
    double c = 0.0;
    for (auto& sw : sweeps) {
        for (uint32_t q = 0; q < n && (uint32_t)__builtin_popcountll(sw.L) < m; ++q) sw.L |= 1ull << q;
        c += k.sweep + k.phase * (double)plan_phases(sw, rb, true).size();
    }
    return c;
}

// Cost-aware local sets for tensor-core plans: each sweep takes the candidate set that
// maximises (gates it runs) x rate - (its launch cost), rate = the cost per gate of a
// reference plan, so a set that runs many gates but needs many phases can lose to one
// that runs slightly fewer in fewer phases.
inline std::vector<Sweep> plan_sweeps_costed(const std::vector<PGate>& gates, uint32_t n, uint32_t m, uint32_t c,
                                             uint32_t rb, double rate, SweepCost cost = COST_TF32) {
    std::vector<Sweep> out;
    std::vector<char> taken(gates.size(), 0);
    size_t first = 0;
    while (first < gates.size()) {
        double best = -1e300;
        uint64_t bestL = 0;
        bool found = false;
        for (uint64_t L : sweep_candidates(gates, taken, first, n, m, c)) {
            std::vector<char> t2 = taken;
            Sweep sw = take_sweep(gates, t2, first, L, n, m);
            if (sw.ops.empty()) continue;
            int got = 0;
            for (size_t k = first; k < gates.size(); ++k) got += (t2[k] && !taken[k]) ? 1 : 0;
            const double score = rate * got - (cost.sweep + cost.phase * (double)plan_phases(sw, rb, true).size());
            if (score > best) {
                best = score;
                bestL = L;
                found = true;
            }
        }
        if (!found) return {};   // no progress (cannot happen with the first-come candidate): give up
        Sweep sw = take_sweep(gates, taken, first, bestL, n, m);
        sw.L = bestL;
        out.push_back(std::move(sw));
        while (first < gates.size() && taken[first]) ++first;
    }
    return out;
}

// Beam search over sweep plans for tensor-core sweeps: breadth-first by sweep, each partial
// plan extended by every candidate local set of sweep_candidates (its phases planned with
// plan_phases), the `width` extensions of highest (gates run) x rate - (modelled cost) kept
// (distinct sets of gates run), extensions that already cost more than the cheapest complete
// plan dropped; returns the cheapest complete plan seen.  rate = the cost per gate of a
// reference plan, as in plan_sweeps_costed.
inline std::vector<Sweep> plan_sweeps_beam(const std::vector<PGate>& gates, uint32_t n, uint32_t m, uint32_t c,
                                           uint32_t rb, double rate, SweepCost cost, size_t width = 16) {
    struct Partial {
        std::vector<char> taken;
        size_t first;
        double cost;
        int done;
        std::vector<uint64_t> sets;
    };
    if (gates.empty()) return {};
    std::vector<Partial> beam(1);
    beam[0].taken.assign(gates.size(), 0);
    beam[0].first = 0;
    beam[0].cost = 0.0;
    beam[0].done = 0;
    double best_cost = 1e300;
    std::vector<uint64_t> best_sets;
    while (!beam.empty()) {
        std::vector<Partial> next;
        std::vector<std::vector<char>> seen;
        for (const Partial& p : beam)
            for (uint64_t L : sweep_candidates(gates, p.taken, p.first, n, m, c)) {
                Partial t{p.taken, p.first, p.cost, p.done, p.sets};
                const Sweep sw = take_sweep(gates, t.taken, p.first, L, n, m);
                if (sw.ops.empty()) continue;
                int got = 0;
                for (size_t k = p.first; k < gates.size(); ++k) got += (t.taken[k] && !p.taken[k]) ? 1 : 0;
                t.cost += cost.sweep + cost.phase * (double)plan_phases(sw, rb, true).size();
                t.done += got;
                t.sets.push_back(L);
                while (t.first < gates.size() && t.taken[t.first]) ++t.first;
                if (t.cost >= best_cost) continue;
                if (t.first >= gates.size()) {
                    best_cost = t.cost;
                    best_sets = t.sets;
                    continue;
                }
                if (std::find(seen.begin(), seen.end(), t.taken) != seen.end()) continue;
                seen.push_back(t.taken);
                next.push_back(std::move(t));
            }
        std::stable_sort(next.begin(), next.end(), [rate](const Partial& a, const Partial& b) {
            return a.done * rate - a.cost > b.done * rate - b.cost;
        });
        if (next.size() > width) next.resize(width);
        beam = std::move(next);
    }
    // replay the chosen local sets into sweeps (as plan_sweeps_costed builds them)
    std::vector<Sweep> out;
    std::vector<char> taken(gates.size(), 0);
    size_t first = 0;
    for (uint64_t L : best_sets) {
        Sweep sw = take_sweep(gates, taken, first, L, n, m);
        sw.L = L;
        out.push_back(std::move(sw));
        while (first < gates.size() && taken[first]) ++first;
    }
    if (first < gates.size()) return {};   // cannot happen: the chosen plan ran every gate
    return out;
}

// The sweep plan.  CUDA-core plans: the first-come and lookahead plans, keeping the one
// with fewer sweeps (each sweep is a full read and write of the state; first-come on a
// tie).  Tensor-core plans (all_slots, five register slots): also the cost-aware and the
// beam-search plans, keeping the plan of least modelled cost (the fewest-sweeps plan on a
// tie, then the cost-aware one).  A gate qubit that stays outside a sweep's
// local set is uniform over each tile, for CUDA-core and tensor-core plans alike.
inline std::vector<Sweep> plan_sweeps(const std::vector<PGate>& gates, uint32_t n, uint32_t m, uint32_t c,
                                      bool all_slots = false, SweepCost k = COST_TF32) {
    auto a = plan_sweeps_first_come(gates, n, m, c);
    auto b = plan_sweeps_lookahead(gates, n, m, c);
    auto best = b.size() < a.size() ? b : a;
    if (!all_slots || gates.empty()) return best;
    const uint32_t rb = 5;
    const double cost_best = plan_cost(best, n, m, rb, k);
    const double rate = cost_best / (double)gates.size();
    auto d = plan_sweeps_costed(gates, n, m, c, rb, rate, k);
    double cost_d = d.empty() ? 1e300 : plan_cost(d, n, m, rb, k);
    auto e = plan_sweeps_beam(gates, n, m, c, rb, rate, k);
    const double cost_e = e.empty() ? 1e300 : plan_cost(e, n, m, rb, k);
    if (cost_e < cost_best && cost_e < cost_d) return e;
    if (cost_d < cost_best) return d;
    return best;
}

inline bool to_pgates(const rq_gate* gates, uint64_t n, std::vector<PGate>& out) {
    const double s2 = 0.70710678118654752440;
    for (uint64_t k = 0; k < n; ++k) {
        const rq_gate& g = gates[k];
        PGate p{};
        p.q0 = g.q0;
        p.q1 = g.q1;
        double h = g.angle / 2.0;
        switch (g.kind) {
            case RQ_GATE_CNOT: p.type = OP_CX; out.push_back(p); break;
            case RQ_GATE_CZ: p.type = OP_CZ; out.push_back(p); break;
            case RQ_GATE_RZZ:
                p.type = OP_ZZ;
                p.m[0] = std::cos(-h); p.m[1] = std::sin(-h); p.m[2] = std::cos(h); p.m[3] = std::sin(h);
                out.push_back(p);
                break;
            case RQ_GATE_SWAP: {
                PGate a{}; a.type = OP_CX; a.q0 = g.q0; a.q1 = g.q1;
                PGate b{}; b.type = OP_CX; b.q0 = g.q1; b.q1 = g.q0;
                out.push_back(a); out.push_back(b); out.push_back(a);
                break;
            }
            case RQ_GATE_Z: p.type = OP_D1; p.m[0] = 1; p.m[2] = -1; p.m[3] = -0.0; out.push_back(p); break;
            case RQ_GATE_S: p.type = OP_D1; p.m[0] = 1; p.m[3] = 1; out.push_back(p); break;
            case RQ_GATE_SDG: p.type = OP_D1; p.m[0] = 1; p.m[2] = -0.0; p.m[3] = -1; out.push_back(p); break;
            case RQ_GATE_T: p.type = OP_D1; p.m[0] = 1; p.m[2] = s2; p.m[3] = s2; out.push_back(p); break;
            case RQ_GATE_TDG: p.type = OP_D1; p.m[0] = 1; p.m[2] = s2; p.m[3] = -s2; out.push_back(p); break;
            case RQ_GATE_RZ:
                p.type = OP_D1;
                p.m[0] = std::cos(-h); p.m[1] = std::sin(-h); p.m[2] = std::cos(h); p.m[3] = std::sin(h);
                out.push_back(p);
                break;
            case RQ_GATE_PHASE:
                p.type = OP_D1; p.m[0] = 1; p.m[2] = std::cos(g.angle); p.m[3] = std::sin(g.angle);
                out.push_back(p);
                break;
            case RQ_GATE_H: { p.type = OP_U1; double m[8] = {s2, 0, s2, 0, s2, 0, -s2, -0.0}; std::memcpy(p.m, m, sizeof m); out.push_back(p); break; }
            case RQ_GATE_X: { p.type = OP_U1; double m[8] = {0, 0, 1, 0, 1, 0, 0, 0}; std::memcpy(p.m, m, sizeof m); out.push_back(p); break; }
            case RQ_GATE_Y: { p.type = OP_U1; double m[8] = {0, 0, -0.0, -1, 0, 1, 0, 0}; std::memcpy(p.m, m, sizeof m); out.push_back(p); break; }
            case RQ_GATE_RX: {
                double c = std::cos(h), sn = -std::sin(h);
                p.type = OP_U1; double m[8] = {c, 0, 0, sn, 0, sn, c, 0}; std::memcpy(p.m, m, sizeof m); out.push_back(p);
                break;
            }
            case RQ_GATE_RY: {
                double c = std::cos(h), sn = std::sin(h);
                p.type = OP_U1; double m[8] = {c, 0, -sn, 0, sn, 0, c, 0}; std::memcpy(p.m, m, sizeof m); out.push_back(p);
                break;
            }
            case RQ_GATE_UNITARY1Q: p.type = OP_U1; std::memcpy(p.m, g.m, sizeof p.m); out.push_back(p); break;
            default: return false;
        }
    }
    return true;
}


// Shared-memory swizzle of a tile element index: XOR the element's column
// inside its 128-byte row with a fold of the row index.  Linear over GF(2),
// so swz(a | b) = swz(a) ^ swz(b) for disjoint bit sets; the kernels combine
// host-swizzled table entries with one per-thread term by XOR.
inline uint32_t swz_host(uint32_t e, uint32_t cb) {
    uint32_t r = e >> cb;
    uint32_t f = r ^ (r >> cb) ^ (r >> (2 * cb)) ^ (r >> (3 * cb));
    return e ^ (f & ((1u << cb) - 1));
}

// Shared-memory layout of the FP16 tensor-core sweeps (complex f32, at most 14 local bits):
// element e is stored at swz16(e) = e ^ g(e), where local bits 0..3 address the 16 8-byte
// units of a 128-byte row and every higher local bit b flips the unit index by its own
// 4-bit pattern SWZ16_ROW[b - 4].  All 14 patterns (with 1, 2, 4, 8 for bits 0..3) are
// distinct and non-zero, so any 8 local bits span all 16 units (8 distinct non-zero vectors
// cannot lie in a 3-dimensional subspace, which holds only 7): a phase can always give its
// warp lanes 5 thread bits whose patterns span the units, and then the 32 8-byte accesses of
// a warp fall on every bank exactly twice (two wavefronts, no conflict), whichever 5 local
// bits the phase keeps in registers.
// SWZ16_ROW nibble k = the pattern of local bit 4 + k: 3, 5, 6, 9, 10, 12, 7, 11, 13, 14
constexpr uint64_t SWZ16_ROW = 0xEDB7CA9653ull;

__host__ __device__ inline uint32_t swz16(uint32_t e) {
    uint32_t g = 0;
    for (int b = 0; b < 10; ++b)
        if ((e >> (4 + b)) & 1u) g ^= (uint32_t)(SWZ16_ROW >> (4 * b)) & 15u;
    return e ^ g;
}

inline uint32_t swz16_unit(uint32_t local_bit) { return swz16(1u << local_bit) & 15u; }

// Re-table a tensor-core program for the FP16 sweep kernel: slot and vector offsets under
// swz16, and per phase an order of the thread bits whose first five (the warp lanes) span all
// 16 bank units (a greedy basis, lowest local bits first), with the thread bits' swizzled
// offsets in tsw.
inline void retable_f16(std::vector<SweepDesc>& descs, std::vector<PhaseDesc>& phases, uint32_t rb) {
    for (auto& d : descs) {
        const uint32_t t = d.m - rb;
        for (uint32_t j = 0; j < (1u << rb) / 2; ++j) d.sgj[j] = swz16(j * (1u << t) * 2u);
    }
    for (auto& ph : phases) {
        for (uint32_t i = 0; i < (1u << rb); ++i) ph.slut[i] = swz16(ph.lut[i]);
        const uint32_t nt = ph.nt;
        std::vector<uint32_t> order, rest;
        uint32_t span[16] = {0};   // reduced basis by leading bit
        for (uint32_t b = 0; b < nt; ++b) {
            uint32_t v = swz16_unit(ph.tbit_local[b]);
            for (int k = 3; k >= 0 && v; --k)
                if ((v >> k) & 1u) {
                    if (span[k]) v ^= span[k];
                    else { span[k] = v; v = 0; order.push_back(b); break; }
                }
            if (order.empty() || order.back() != b) rest.push_back(b);
        }
        for (uint32_t b : rest) order.push_back(b);
        uint8_t tl[12], tg[12];
        for (uint32_t b = 0; b < nt; ++b) {
            tl[b] = ph.tbit_local[order[b]];
            tg[b] = ph.tbit_global[order[b]];
        }
        for (uint32_t b = 0; b < nt; ++b) {
            ph.tbit_local[b] = tl[b];
            ph.tbit_global[b] = tg[b];
        }
        for (uint32_t b = 0; b < 8; ++b) ph.tsw[b] = b < nt ? (uint16_t)swz16(1u << ph.tbit_local[b]) : 0;
    }
}

// Flatten sweeps into kernel tables: one SweepDesc per sweep, PhaseDescs,
// op records and the f64 matrix entries (narrowed later for f32 states).
// given_phases (optional): the phase plans to use per sweep instead of planning them (a program
// rebuilt for new gate values with an unchanged structure); used_phases (optional) receives the
// phase plans of every sweep.
inline void build_program(std::vector<Sweep>& sweeps, uint32_t nq, uint32_t m, uint32_t c, uint32_t rb,
                          uint32_t epv, std::vector<SweepDesc>& descs, std::vector<PhaseDesc>& phases,
                          std::vector<SwOp>& ops, std::vector<double>& mats, bool all_slots = false,
                          const std::vector<std::vector<PhasePlan>>* given_phases = nullptr,
                          std::vector<std::vector<PhasePlan>>* used_phases = nullptr) {
    size_t sweep_index = 0;
    for (auto& sw : sweeps) {
        uint64_t L = sw.L;
        for (uint32_t q = 0; q < nq && (uint32_t)__builtin_popcountll(L) < m; ++q) L |= 1ull << q;
        sw.L = L;
        SweepDesc d{};
        d.n = nq;
        d.m = m;
        d.c = c;
        uint32_t li = 0, ni = 0;
        uint8_t local_index[64];
        for (uint32_t q = 0; q < nq; ++q) {
            if ((L >> q) & 1) { local_index[q] = (uint8_t)li; d.local_global[li++] = (uint8_t)q; }
            else d.nonlocal[ni++] = (uint8_t)q;
        }
        d.nonlocal_count = ni;
        const uint32_t t = m - rb;
        const uint32_t VPT = (1u << rb) / epv;
        const uint32_t cb = epv == 2 ? 4 : 3;
        for (uint32_t j = 0; j < VPT; ++j) {
            uint64_t x = (uint64_t)j * (1ull << t) * epv, gsum = 0;
            for (uint32_t b = 0; b < m; ++b)
                if ((x >> b) & 1) gsum |= 1ull << d.local_global[b];
            d.gj[j] = gsum;
            d.sgj[j] = swz_host((uint32_t)x, cb);
        }
        d.phase_begin = (uint32_t)phases.size();
        auto pplan = given_phases ? (*given_phases)[sweep_index] : plan_phases(sw, rb, all_slots);
        if (used_phases) used_phases->push_back(pplan);
        ++sweep_index;
        for (auto& pp : pplan) {
            PhaseDesc Ph{};
            Ph.op_begin = (uint32_t)ops.size();
            int slot_of[64];
            for (int q = 0; q < 64; ++q) slot_of[q] = -1;
            uint32_t slots[RBMAX], ns = 0;
            for (uint32_t q = 0; q < nq; ++q)
                if ((pp.R >> q) & 1) { slot_of[q] = (int)ns; slots[ns++] = q; }
            uint32_t nt = 0;
            for (uint32_t b = 0; b < m; ++b) {
                uint32_t q = d.local_global[b];
                if (!((pp.R >> q) & 1)) { Ph.tbit_local[nt] = (uint8_t)b; Ph.tbit_global[nt] = (uint8_t)q; ++nt; }
            }
            Ph.nt = nt;
            for (uint32_t i = 0; i < (1u << rb); ++i) {
                uint32_t off = 0;
                for (uint32_t sidx = 0; sidx < ns; ++sidx)
                    if ((i >> sidx) & 1) off |= 1u << local_index[slots[sidx]];
                Ph.lut[i] = (uint16_t)off;
                Ph.slut[i] = swz_host(off, cb);
            }
            for (uint32_t sidx = 0; sidx < ns; ++sidx) Ph.slot_global[sidx] = (uint8_t)slots[sidx];
            for (int oi : pp.ops) {
                const PGate& g = sw.ops[oi];
                SwOp o{};
                o.type = g.type;
                o.q0 = (uint8_t)g.q0;
                o.q1 = (uint8_t)g.q1;
                o.k0 = (int8_t)slot_of[g.q0];
                o.k1 = (g.type == OP_CX || g.type == OP_CZ || g.type == OP_ZZ) ? (int8_t)slot_of[g.q1] : -1;
                o.param = g.param;
                o.mat = (uint32_t)(mats.size() / 2);
                int cnt = g.type == OP_U1 ? 8 : (g.type == OP_D1 || g.type == OP_ZZ) ? 4 : 0;
                for (int k = 0; k < cnt; ++k) mats.push_back(g.m[k]);
                ops.push_back(o);
            }
            Ph.op_end = (uint32_t)ops.size();
            phases.push_back(Ph);
        }
        d.phase_end = (uint32_t)phases.size();
        descs.push_back(d);
    }
    if (mats.empty()) mats.push_back(0.0);
    if (ops.empty()) ops.push_back(SwOp{});
    if (phases.empty()) phases.push_back(PhaseDesc{});
}

// ---- dense fusion for the tensor cores ----------------------------------
//
// In a phase every thread holds the 32 amplitudes spanned by the five register
// slots, so any run of ops that only reads and writes slot bits is one 32x32
// complex matrix, the same for every thread.  fuse_dense rewrites each phase:
// ops touching a non-slot bit (a CNOT controlled by a thread bit, a diagonal
// on a thread bit) are deferred past the slot-local ops that do not share a
// qubit with them (gates on disjoint qubits commute), the slot-local ops
// become one OP_DENSE when there are at least `min_ops` of them, and the
// deferred ops follow in their original order.
//
// Operand image of a dense op, as the MMA's B operand: B[c][k] (c = output
// 2i'+r', k = input 2i+r, r = 0 real / 1 imaginary part) is the real form of
// U: B[2i'][2i] = Re U, B[2i'][2i+1] = -Im U, B[2i'+1][2i] = Im U,
// B[2i'+1][2i+1] = Re U, stored in the no-swizzle K-major core-matrix layout
// (element (c, k) at byte (c/8)*2048 + (k/4)*128 + (c%8)*16 + (k%4)*4), as a
// TF32 high part followed by the FP32 remainder (16 KB each).
constexpr int DENSE_FLOATS = 64 * 64;          // one 64x64 operand image
constexpr int DENSE_IMAGE_FLOATS = 2 * DENSE_FLOATS;

// FP16 operand images (RQ_EXEC_SWEEP_TC16): the same B, scaled by 2^DENSE_F16_SCALE_LOG2,
// split into an FP16 high part h = fp16(B') and low part l = fp16(B' - h) (both rounded to
// nearest even from the f64 product), each 64x64 in the no-swizzle K-major core-matrix
// layout of 16-bit elements: element (c, k) at byte (c/8)*1024 + (k/8)*128 + (c%8)*16 +
// (k%8)*2; high part then low part, 8 KB each.
constexpr int DENSE_F16_SCALE_LOG2 = 14;
constexpr int DENSE_F16_WORDS = 64 * 64;       // 32-bit words per image (two 8 KB parts)

enum DenseFormat : int { DENSE_TF32 = 0, DENSE_F16 = 1 };
inline size_t dense_image_words(int fmt) { return fmt == DENSE_F16 ? DENSE_F16_WORDS : DENSE_IMAGE_FLOATS; }

// Exactly rounded double arithmetic, the same on the host and the device (no fused
// multiply-add on either side), so that operand images built on the GPU are bit-identical to
// the host's restatement of the same products.
__host__ __device__ inline double dmul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ inline double dadd(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ inline double dsub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}

// v <- op(v) on a 32-vector of register amplitudes (the kernel's op semantics); u0 / u1
// are the values of q0 / q1 when they are not register slots (uniform over a tile)
__host__ __device__ inline void apply_op32(const SwOp& o, const double* mt, double* v /* 64: re, im */,
                                           int u0 = 0, int u1 = 0) {
    if (o.type == OP_U1) {
        const int b = 1 << o.k0;
        for (int i = 0; i < 32; ++i) {
            if (i & b) continue;
            const int j = i | b;
            const double xr = v[2 * i], xi = v[2 * i + 1], yr = v[2 * j], yi = v[2 * j + 1];
            v[2 * i] = dsub(dadd(dsub(dmul(mt[0], xr), dmul(mt[1], xi)), dmul(mt[2], yr)), dmul(mt[3], yi));
            v[2 * i + 1] = dadd(dadd(dadd(dmul(mt[0], xi), dmul(mt[1], xr)), dmul(mt[2], yi)), dmul(mt[3], yr));
            v[2 * j] = dsub(dadd(dsub(dmul(mt[4], xr), dmul(mt[5], xi)), dmul(mt[6], yr)), dmul(mt[7], yi));
            v[2 * j + 1] = dadd(dadd(dadd(dmul(mt[4], xi), dmul(mt[5], xr)), dmul(mt[6], yi)), dmul(mt[7], yr));
        }
    } else if (o.type == OP_D1 || o.type == OP_ZZ) {
        for (int i = 0; i < 32; ++i) {
            bool second;
            if (o.type == OP_D1) {
                second = (o.k0 >= 0 ? (i >> o.k0) & 1 : u0) != 0;
            } else {   // diag(en, ep, ep, en): the second entry for differing bits
                const int b0 = o.k0 >= 0 ? (i >> o.k0) & 1 : u0, b1 = o.k1 >= 0 ? (i >> o.k1) & 1 : u1;
                second = (b0 ^ b1) != 0;
            }
            const double dr = second ? mt[2] : mt[0], di = second ? mt[3] : mt[1];
            const double xr = v[2 * i], xi = v[2 * i + 1];
            v[2 * i] = dsub(dmul(xr, dr), dmul(xi, di));
            v[2 * i + 1] = dadd(dmul(xr, di), dmul(xi, dr));
        }
    } else if (o.type == OP_CX) {
        const int t = 1 << o.k1;
        for (int i = 0; i < 32; ++i)
            if (!(i & t) && (o.k0 >= 0 ? (i >> o.k0) & 1 : u0)) {
                const double ar = v[2 * i], ai = v[2 * i + 1];
                v[2 * i] = v[2 * (i | t)];
                v[2 * i + 1] = v[2 * (i | t) + 1];
                v[2 * (i | t)] = ar;
                v[2 * (i | t) + 1] = ai;
            }
    } else if (o.type == OP_CZ) {
        for (int i = 0; i < 32; ++i) {
            const int b0 = o.k0 >= 0 ? (i >> o.k0) & 1 : u0, b1 = o.k1 >= 0 ? (i >> o.k1) & 1 : u1;
            if (b0 && b1) {
                v[2 * i] = -v[2 * i];
                v[2 * i + 1] = -v[2 * i + 1];
            }
        }
    }
}

__host__ __device__ inline float tf32_round(float x) {
#ifdef __CUDA_ARCH__
    uint32_t b = __float_as_uint(x);
#else
    uint32_t b;
    std::memcpy(&b, &x, 4);
#endif
    if ((b & 0x7F800000u) != 0x7F800000u) {   // finite: round to nearest, ties away, at 10 mantissa bits
        b += 0x1000u;
        b &= 0xFFFFE000u;
    }
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float r;
    std::memcpy(&r, &b, 4);
    return r;
#endif
}

__host__ __device__ inline size_t dense_offset(int c, int k) {   // in floats
    return (size_t)(c / 8) * 512 + (size_t)(k / 4) * 32 + (size_t)(c % 8) * 4 + (size_t)(k % 4);
}

// IEEE binary16 bits of x, rounded to nearest even (subnormals kept; |x| < 65520 here)
__host__ __device__ inline uint16_t f16_bits(double x) {
    const uint16_t sign = signbit(x) ? 0x8000u : 0u;
    const double a = fabs(x);
    if (a == 0.0) return sign;
    if (a >= 65520.0) return (uint16_t)(sign | 0x7C00u);
    int e = 0;
    const double m = frexp(a, &e);   // a = m * 2^e, m in [0.5, 1)
    int E = e - 1;                   // a = (2m) * 2^E
    if (E < -14) return (uint16_t)(sign | (uint16_t)nearbyint(a * 16777216.0));   // units of 2^-24
    double q = nearbyint(m * 2048.0);   // 11 significant bits, in [1024, 2048]
    if (q == 2048.0) { q = 1024.0; E += 1; }
    if (E > 15) return (uint16_t)(sign | 0x7C00u);
    return (uint16_t)(sign | (uint16_t)(((E + 15) << 10) | ((int)q - 1024)));
}

__host__ __device__ inline double f16_value(uint16_t h) {
    const int e = (h >> 10) & 0x1F, f = h & 0x3FF;
    double v = e == 0 ? ldexp((double)f, -24) : ldexp((double)(1024 + f), e - 25);
    return (h & 0x8000u) ? -v : v;
}

__host__ __device__ inline size_t dense_offset16(int c, int k) {   // in 16-bit elements
    return (size_t)(c / 8) * 512 + (size_t)(k / 8) * 64 + (size_t)(c % 8) * 8 + (size_t)(k % 8);
}

// Column col of an operand image from u = U e_col (32 complex, re/im interleaved): the entries
// B[2i'+r'][2col+r] of the real form of U, split into the format's high and low parts.
__host__ __device__ inline void dense_image_column(const double* u, int col, uint32_t* out_words, int fmt) {
    const double sc = fmt == DENSE_F16 ? (double)(1u << DENSE_F16_SCALE_LOG2) : 1.0;
    for (int i = 0; i < 32; ++i) {
        const double ur = u[2 * i], ui = u[2 * i + 1];
        const double vals[2][2] = {{ur, -ui}, {ui, ur}};
        for (int rp = 0; rp < 2; ++rp)
            for (int r = 0; r < 2; ++r) {
                if (fmt == DENSE_F16) {
                    uint16_t* out = reinterpret_cast<uint16_t*>(out_words);
                    const double x = dmul(vals[rp][r], sc);
                    const uint16_t hi = f16_bits(x);
                    const uint16_t lo = f16_bits(dsub(x, f16_value(hi)));
                    const size_t off = dense_offset16(2 * i + rp, 2 * col + r);
                    out[off] = hi;
                    out[DENSE_F16_WORDS + off] = lo;
                } else {
                    float* out = reinterpret_cast<float*>(out_words);
                    const double x = vals[rp][r];
                    const float hi = tf32_round((float)x);
                    const float lo = (float)dsub(x, (double)hi);
                    const size_t off = dense_offset(2 * i + rp, 2 * col + r);
                    out[off] = hi;
                    out[DENSE_FLOATS + off] = lo;
                }
            }
    }
}

// Tensor-core plans: every phase becomes one OP_DENSE.  Gate qubits that are register
// slots index the 32-dimensional space; the other gate qubits are outside the sweep's local
// set (the phase planner makes every local gate qubit a slot), so their values are fixed
// for a whole tile.  For the at most DENSE_MAX_VQ such qubits of a phase one image is built
// per value assignment (variant v: bit j of v = value of the j-th qubit); the kernel picks
// the variant from the tile's index bits.  Returns false when a phase needs more.
constexpr int DENSE_MAX_VQ = 5;

__host__ __device__ inline int dense_nvq(const SwOp& o) { return o.k0; }
__host__ __device__ inline uint32_t dense_vq(const SwOp& o, int j) {
    switch (j) {
        case 0: return o.q0;
        case 1: return o.q1;
        case 2: return o.pad;
        case 3: return o.pad2 & 0xFFu;
        default: return (o.pad2 >> 8) & 0xFFu;
    }
}

// One operand image to build: a (phase, variant) pair -- the image slot, the phase's range in
// the op list before fusion, and the values of its qubits outside the tile.
struct DenseJob {
    uint32_t slot, op_begin, op_end, var, nvq;
    uint32_t vq[DENSE_MAX_VQ];
};

// Column col of the job's 32x32 unitary: the phase's ops applied in order to e_col.
__host__ __device__ inline void dense_job_column(const DenseJob& jb, const SwOp* ops, const double* mats, int col,
                                                 double* v /* 64 */) {
    for (int k = 0; k < 64; ++k) v[k] = 0.0;
    v[2 * col] = 1.0;
    for (uint32_t o = jb.op_begin; o < jb.op_end; ++o) {
        const SwOp& op = ops[o];
        int u0 = 0, u1 = 0;
        for (uint32_t k = 0; k < jb.nvq; ++k) {
            if (jb.vq[k] == op.q0) u0 = (int)((jb.var >> k) & 1u);
            if (jb.vq[k] == op.q1) u1 = (int)((jb.var >> k) & 1u);
        }
        apply_op32(op, mats + 2 * (size_t)op.mat, v, u0, u1);
    }
}

// Rewrites every phase into one OP_DENSE (its image slots and outside qubits), leaving in
// *jobs the images to build and in *pre_ops the op list they read (the ops before fusion);
// with build_images the images are built here, on the host's cores, else the caller builds
// them (the library does so on the GPU, bit-identically).  Returns false when a phase cannot
// be one dense op.
inline bool fuse_dense(std::vector<SweepDesc>& descs, std::vector<PhaseDesc>& phases, std::vector<SwOp>& ops,
                       const std::vector<double>& mats, std::vector<uint32_t>& images, uint64_t* ndense,
                       int fmt = DENSE_TF32, std::vector<DenseJob>* jobs_out = nullptr,
                       std::vector<SwOp>* pre_ops = nullptr, bool build_images = true) {
    const size_t words = dense_image_words(fmt);
    std::vector<SwOp> out;
    std::vector<uint32_t> sweep_of(phases.size(), 0);
    for (size_t d = 0; d < descs.size(); ++d) {
        for (uint32_t p = descs[d].phase_begin; p < descs[d].phase_end; ++p) sweep_of[p] = (uint32_t)d;
        descs[d].img_begin = 0;
        descs[d].img_count = 0;
    }
    std::vector<DenseJob> jobs;
    size_t nimg = 0;
    for (size_t pi = 0; pi < phases.size(); ++pi) {
        auto& ph = phases[pi];
        SweepDesc& sd = descs[sweep_of[pi]];
        // the phase's tile-uniform qubits, in first-use order
        std::vector<uint32_t> vq;
        auto note = [&](int k, uint32_t q) {
            if (k < 0 && std::find(vq.begin(), vq.end(), q) == vq.end()) vq.push_back(q);
        };
        for (uint32_t o = ph.op_begin; o < ph.op_end; ++o) {
            const SwOp& op = ops[o];
            switch (op.type) {
                case OP_U1: if (op.k0 < 0) return false; break;
                case OP_D1: note(op.k0, op.q0); break;
                case OP_CX: if (op.k1 < 0) return false; note(op.k0, op.q0); break;
                case OP_CZ: case OP_ZZ: note(op.k0, op.q0); note(op.k1, op.q1); break;
                default: return false;
            }
        }
        if (vq.size() > (size_t)DENSE_MAX_VQ) return false;
        const size_t first = nimg;
        const uint32_t nvar = 1u << vq.size();
        for (uint32_t var = 0; var < nvar; ++var) {
            DenseJob jb{};
            jb.slot = (uint32_t)nimg++;
            jb.op_begin = ph.op_begin;
            jb.op_end = ph.op_end;
            jb.var = var;
            jb.nvq = (uint32_t)vq.size();
            for (size_t k = 0; k < vq.size(); ++k) jb.vq[k] = vq[k];
            jobs.push_back(jb);
        }
        if (sd.img_count == 0) sd.img_begin = (uint32_t)first;
        sd.img_count += nvar;
        SwOp d{};
        d.type = OP_DENSE;
        d.k0 = (int8_t)vq.size();
        d.k1 = -1;
        uint8_t b[5] = {0, 0, 0, 0, 0};
        for (size_t k = 0; k < vq.size(); ++k) b[k] = (uint8_t)vq[k];
        d.q0 = b[0];
        d.q1 = b[1];
        d.pad = b[2];
        d.pad2 = (uint32_t)b[3] | ((uint32_t)b[4] << 8);
        d.mat = (uint32_t)first;
        const uint32_t begin = (uint32_t)out.size();
        out.push_back(d);
        ph.op_begin = begin;
        ph.op_end = (uint32_t)out.size();
        ++*ndense;
    }
    images.assign(nimg * words, 0u);
    if (build_images) {
        auto work = [&](size_t j0, size_t j1) {
            double v[64];
            for (size_t jj = j0; jj < j1; ++jj)
                for (int col = 0; col < 32; ++col) {
                    dense_job_column(jobs[jj], ops.data(), mats.data(), col, v);
                    dense_image_column(v, col, images.data() + (size_t)jobs[jj].slot * words, fmt);
                }
        };
        const size_t nt =
            std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), (jobs.size() + 15) / 16));
        if (nt <= 1) {
            work(0, jobs.size());
        } else {
            std::vector<std::thread> pool;
            const size_t per = (jobs.size() + nt - 1) / nt;
            for (size_t t = 0; t < nt; ++t) {
                const size_t j0 = t * per, j1 = std::min(jobs.size(), j0 + per);
                if (j0 < j1) pool.emplace_back(work, j0, j1);
            }
            for (auto& th : pool) th.join();
        }
    }
    if (jobs_out) jobs_out->swap(jobs);
    if (out.empty()) out.push_back(SwOp{});
    if (pre_ops) *pre_ops = ops;
    ops.swap(out);
    return true;
}

}  // namespace rqp

