// Host check of the sweep and phase planners of rq_plan.cuh (no GPU needed).
//
// Random circuits are planned with every planner combination (first-come,
// lookahead, cost-aware and beam-search sweeps, first-come, lookahead and beam-search phases, CUDA-core and
// tensor-core slot rules); the planned ops are applied in plan order (sweep, phase, op) to a
// state vector in double precision, which must equal the gates applied in list
// order.  The planners' own rules are checked on the way: every op's required
// qubits are local and on slots, slot sets fit the register count, tensor-core
// phases keep every local gate qubit on a slot and at most four qubits outside.
// Exit status 0 = all good; the first failure is printed.
#include "rq_plan.cuh"

#include <complex>
#include <cstdio>
#include <random>

using namespace rqp;
using Cx = std::complex<double>;

static void apply(std::vector<Cx>& a, const PGate& g) {
    const uint64_t N = a.size();
    const uint64_t b0 = 1ull << g.q0, b1 = 1ull << g.q1;
    switch (g.type) {
        case OP_U1: {
            const Cx m00(g.m[0], g.m[1]), m01(g.m[2], g.m[3]), m10(g.m[4], g.m[5]), m11(g.m[6], g.m[7]);
            for (uint64_t i = 0; i < N; ++i)
                if (!(i & b0)) {
                    const Cx x = a[i], y = a[i | b0];
                    a[i] = m00 * x + m01 * y;
                    a[i | b0] = m10 * x + m11 * y;
                }
            break;
        }
        case OP_D1:
            for (uint64_t i = 0; i < N; ++i) a[i] *= (i & b0) ? Cx(g.m[2], g.m[3]) : Cx(g.m[0], g.m[1]);
            break;
        case OP_CX:
            for (uint64_t i = 0; i < N; ++i)
                if ((i & b0) && !(i & b1)) std::swap(a[i], a[i | b1]);
            break;
        case OP_CZ:
            for (uint64_t i = 0; i < N; ++i)
                if ((i & b0) && (i & b1)) a[i] = -a[i];
            break;
        case OP_ZZ:
            for (uint64_t i = 0; i < N; ++i)
                a[i] *= (!(i & b0) == !(i & b1)) ? Cx(g.m[0], g.m[1]) : Cx(g.m[2], g.m[3]);
            break;
        default:
            std::printf("unexpected op type %d\n", (int)g.type);
            std::exit(2);
    }
}

static std::vector<rq_gate> random_circuit(uint32_t n, std::mt19937_64& r, bool brickwork) {
    std::vector<rq_gate> out;
    std::uniform_real_distribution<double> ang(0.0, 6.283185307179586);
    const int kinds1[] = {RQ_GATE_H, RQ_GATE_X, RQ_GATE_Y, RQ_GATE_Z, RQ_GATE_S, RQ_GATE_T, RQ_GATE_RX,
                          RQ_GATE_RY, RQ_GATE_RZ, RQ_GATE_PHASE};
    const int kinds2[] = {RQ_GATE_CNOT, RQ_GATE_CZ, RQ_GATE_RZZ, RQ_GATE_SWAP};
    if (brickwork) {
        for (int l = 0; l < 8; ++l) {
            for (uint32_t q = 0; q < n; ++q) {
                rq_gate z{}; z.kind = RQ_GATE_RZ; z.q0 = q; z.angle = ang(r); out.push_back(z);
                rq_gate x{}; x.kind = RQ_GATE_RX; x.q0 = q; x.angle = ang(r); out.push_back(x);
            }
            for (uint32_t q = l & 1; q + 1 < n; q += 2) {
                rq_gate c{}; c.kind = RQ_GATE_CNOT; c.q0 = q; c.q1 = q + 1; out.push_back(c);
            }
        }
        return out;
    }
    const int count = 60 + (int)(r() % 120);
    for (int k = 0; k < count; ++k) {
        rq_gate g{};
        g.angle = ang(r);
        g.q0 = (uint32_t)(r() % n);
        if (r() % 3 == 0) {
            g.kind = kinds2[r() % 4];
            do g.q1 = (uint32_t)(r() % n); while (g.q1 == g.q0);
        } else {
            g.kind = kinds1[r() % 10];
        }
        out.push_back(g);
    }
    return out;
}

static int fail(const char* what, int trial) {
    std::printf("trial %d: %s\n", trial, what);
    return 1;
}

int main() {
    std::mt19937_64 r(12345);
    int trials = 0;
    for (int trial = 0; trial < 240; ++trial) {
        const uint32_t n = 8 + (uint32_t)(trial % 5);          // 8..12 qubits
        const uint32_t m = 6 + (uint32_t)(trial % 3);          // 6..8 local
        const uint32_t c = 3;
        const bool brick = (trial % 4) == 0;
        const auto circ = random_circuit(n, r, brick);
        std::vector<PGate> pg;
        if (!to_pgates(circ.data(), circ.size(), pg)) return fail("to_pgates", trial);
        std::vector<Cx> want((size_t)1 << n);
        std::normal_distribution<double> nd;
        for (auto& v : want) v = Cx(nd(r), nd(r));
        const std::vector<Cx> start = want;
        for (const auto& g : pg) apply(want, g);
        for (int sp = 0; sp < 7; ++sp) {
            std::vector<Sweep> sweeps = sp == 0 ? plan_sweeps_first_come(pg, n, m, c)
                                      : sp == 1 ? plan_sweeps_lookahead(pg, n, m, c)
                                      : sp == 2 ? plan_sweeps(pg, n, m, c)
                                      : sp == 3 ? plan_sweeps(pg, n, m, c, true)
                                      : sp == 4 ? plan_sweeps(pg, n, m, c, true, COST_F16)
                                      : sp == 5 ? plan_sweeps_costed(pg, n, m, c, 5, 0.05)
                                                : plan_sweeps_beam(pg, n, m, c, 5, 0.05, COST_F16);
            if (sp >= 3 && sp != 5 && !pg.empty()) {   // tensor-core plans: never above the fewest-sweeps plan's cost
                auto a = plan_sweeps_first_come(pg, n, m, c), b = plan_sweeps_lookahead(pg, n, m, c);
                const double ref = plan_cost(b.size() < a.size() ? b : a, n, m, 5, COST_F16);
                if (sp == 4 && plan_cost(sweeps, n, m, 5, COST_F16) > ref + 1e-9)
                    return fail("plan_sweeps costs more than the fewest-sweeps plan", trial);
            }
            if (sweeps.empty() && !pg.empty()) return fail("no sweep plan", trial);
            for (int pp = 0; pp < 4; ++pp)
                for (int tc = 0; tc < 2; ++tc) {
                    const uint32_t rb = tc ? 5 : (trial % 2 ? 5 : 4);
                    std::vector<Cx> a = start;
                    bool gave_up = false;
                    for (Sweep sw : sweeps) {
                        for (uint32_t q = 0; q < n && (uint32_t)__builtin_popcountll(sw.L) < m; ++q) sw.L |= 1ull << q;
                        if ((uint32_t)__builtin_popcountll(sw.L) > m) return fail("sweep has too many local qubits", trial);
                        for (const auto& g : sw.ops)
                            if (needs(g, false) & ~sw.L) return fail("op needs a qubit outside its sweep", trial);
                        const auto phases = pp == 0 ? plan_phases_first_come(sw, rb, tc)
                                            : pp == 1 ? plan_phases_lookahead(sw, rb, tc)
                                            : pp == 2 ? plan_phases_beam(sw, rb, tc)
                                                      : plan_phases(sw, rb, tc);
                        if (phases.empty() && !sw.ops.empty()) {
                            if (pp == 1 || pp == 2) {   // the lookahead and the beam may give up; plan_phases falls back
                                gave_up = true;
                                break;
                            }
                            return fail("no phase plan", trial);
                        }
                        if (pp == 3 && phases.size() > plan_phases_first_come(sw, rb, tc).size())
                            return fail("plan_phases has more phases than the first-come plan", trial);
                        std::vector<int> seen(sw.ops.size(), 0);
                        for (const auto& ph : phases) {
                            if ((uint32_t)__builtin_popcountll(ph.R) > rb) return fail("too many slots", trial);
                            if (ph.R & ~sw.L) return fail("slot outside the tile", trial);
                            uint64_t outside = 0;
                            for (int k : ph.ops) {
                                const PGate& g = sw.ops[k];
                                const uint64_t need = needs(g, false) | (tc ? (qmask(g) & sw.L) : 0ull);
                                if (need & ~ph.R) return fail("op qubit not on a slot", trial);
                                if (tc) outside |= qmask(g) & ~sw.L;
                                ++seen[k];
                                apply(a, g);
                            }
                            if (__builtin_popcountll(outside) > DENSE_MAX_VQ_PLAN) return fail("too many outside qubits", trial);
                        }
                        for (int v : seen)
                            if (v != 1) return fail("op not applied exactly once", trial);
                    }
                    if (gave_up) continue;
                    double err = 0.0;
                    for (size_t i = 0; i < a.size(); ++i) err = std::max(err, std::abs(a[i] - want[i]));
                    if (err > 1e-10) {
                        std::printf("trial %d sweeps %d phases %d tc %d: max error %.3e\n", trial, sp, pp, tc, err);
                        return 1;
                    }
                    ++trials;
                }
        }
    }
    // The FP16 sweep kernel's shared-memory layout (swz16, retable_f16): a bijection on a
    // 13-bit tile; after re-tabling, every phase's (thread, register) pairs still cover the
    // tile exactly once, and the five lane bits of every phase span all 16 bank units (the
    // 32 8-byte accesses of a warp hit each bank exactly twice).
    {
        std::vector<int> hit(1u << 14, 0);
        for (uint32_t e = 0; e < (1u << 14); ++e) ++hit[swz16(e)];
        for (int h : hit)
            if (h != 1) return fail("swz16 is not a bijection", -1);
        for (int t2 = 0; t2 < 60; ++t2) {
            // 13 local bits (256-thread tiles) and 14 (512 threads, the ninth thread bit's
            // offset computed from tbit_local[8] as the kernel does)
            const uint32_t m = t2 % 3 == 2 ? 14 : 13, n = 16 + (uint32_t)(t2 % 5), c = 5, rb = 5;
            const uint32_t tb = m - rb;
            const auto circ = random_circuit(n, r, t2 % 2 == 0);
            std::vector<PGate> pg;
            if (!to_pgates(circ.data(), circ.size(), pg)) return fail("to_pgates", t2);
            auto sweeps = plan_sweeps(pg, n, m, c, true);
            std::vector<SweepDesc> descs;
            std::vector<PhaseDesc> phases;
            std::vector<SwOp> ops;
            std::vector<double> mats;
            build_program(sweeps, n, m, c, rb, 2, descs, phases, ops, mats, true);
            const std::vector<PhaseDesc> before = phases;
            retable_f16(descs, phases, rb);
            for (size_t pi = 0; pi < phases.size(); ++pi) {
                const PhaseDesc& ph = phases[pi];
                uint64_t set_a = 0, set_b = 0;
                for (uint32_t b = 0; b < ph.nt; ++b) {
                    set_a |= 1ull << ph.tbit_local[b];
                    set_b |= 1ull << before[pi].tbit_local[b];
                }
                if (set_a != set_b || ph.nt != tb) return fail("retable changed the thread bits", t2);
                uint32_t basis[4] = {0, 0, 0, 0};
                int rank = 0;
                for (uint32_t b = 0; b < 5; ++b) {
                    uint32_t v = swz16(1u << ph.tbit_local[b]) & 15u;
                    for (int k = 3; k >= 0 && v; --k)
                        if ((v >> k) & 1u) {
                            if (basis[k]) v ^= basis[k];
                            else { basis[k] = v; ++rank; v = 0; }
                        }
                }
                if (rank != 4) return fail("lane bits do not span the banks", t2);
                std::vector<int> cover(1u << m, 0);
                for (uint32_t tid = 0; tid < (1u << tb); ++tid) {
                    uint32_t sb = 0;
                    for (uint32_t b = 0; b < 8; ++b)
                        if ((tid >> b) & 1u) sb ^= ph.tsw[b];
                    if (tb > 8 && ((tid >> 8) & 1u)) sb ^= swz16(1u << ph.tbit_local[8]);
                    for (uint32_t i = 0; i < 32; ++i) ++cover[sb ^ ph.slut[i]];
                }
                for (int v : cover)
                    if (v != 1) return fail("retabled phase does not cover the tile once", t2);
            }
            for (const auto& d : descs)
                for (uint32_t j = 0; j < 16; ++j)
                    if (d.sgj[j] != swz16(j * (1u << tb) * 2u)) return fail("sgj not under swz16", t2);
        }
    }
    {   // the autotuner's pick: a later candidate must win by more than 2 %
        const float ms1[4] = {400.f, 130.f, 100.f, 99.f};   // CUDA cores, 3xTF32, FP16 13, FP16 12
        const bool all[4] = {true, true, true, true};
        if (pick_fastest(ms1, all, 4) != 2) return fail("a 1 % faster later candidate was taken", -1);
        const float ms2[4] = {400.f, 130.f, 100.f, 97.f};
        if (pick_fastest(ms2, all, 4) != 3) return fail("a 3 % faster later candidate was not taken", -1);
        const bool no_tc[4] = {true, false, false, false};
        if (pick_fastest(ms2, no_tc, 4) != 0) return fail("an ineligible candidate was taken", -1);
        const float ms3[3] = {10.f, 10.f, 10.f};
        if (pick_fastest(ms3, all, 3) != 0) return fail("a tie did not keep the first candidate", -1);
    }
    std::printf("ok %d plans\n", trials);
    return 0;
}
