// rq_batch.cu -- batched QAOA-MaxCut: many graphs and parameter sets at once.
//
// The reference evaluates one QAOA circuit at a time: evaluate_qaoa_cost
// (qaoa.rs:179-201) builds the circuit of build_qaoa_circuit (qaoa.rs:125-153:
// H on every qubit, then per layer Rzz(2*gamma*w) on every edge and
// Rx(2*beta) on every qubit), runs it on a fresh state and sums
// w*(1 - <Z_i Z_j>)/2 over the edges with one expectation pass per edge.
// Here every circuit of a batch runs through shared sweep programs:
//
//  * circuits with the same qubit count form a class and share one planned
//    program (rq_plan.cuh); a launch covers (circuit, tile) pairs of a class;
//  * H^n|0> is synthesised by the first sweep (uniform amplitude 2^(-n/2));
//  * the product of all Rzz of a layer is one diagonal phase
//    exp(-i*gamma*(|E| - 2 cut(x))) (unit weights): each thread derives
//    cut(x) for its 2^RB register amplitudes from the graph's neighbour masks
//    (the cut of its fixed bits, one count change per register slot, and the
//    edges between slots) and looks the phase up in a table;
//  * the last sweep reduces <C> = sum_x |a_x|^2 cut(x) in FP64 (the same
//    quantity as the per-edge sum of qaoa.rs:194-200) into per-tile partials;
//  * optional shots: FP64 prefix trees per circuit, then every shot walks its
//    circuit's tree with the documented uniform stream, and a block reduction
//    keeps the best cut (highest cut, lowest shot index on ties).
#include "rq_internal.cuh"
#include "rq_plan.cuh"


#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace {

using rqd::C2;
using namespace rqp;

template <typename T> struct Vec16b;
template <> struct Vec16b<float> { using t = float4; static constexpr int EPV = 2; };
template <> struct Vec16b<double> { using t = double2; static constexpr int EPV = 1; };

template <typename T>
__device__ __forceinline__ uint32_t swzb(uint32_t e) {
    constexpr int CB = sizeof(typename C2<T>::t) == 8 ? 4 : 3;
    uint32_t r = e >> CB;
    uint32_t f = r ^ (r >> CB) ^ (r >> (2 * CB)) ^ (r >> (3 * CB));
    return e ^ (f & ((1u << CB) - 1));
}

// index of the lowest set bit of 1 <= g < 32 (the Gray-code bit that flips at step g)
__host__ __device__ constexpr int gray_bit(int g) { return (g & 1) ? 0 : (g & 2) ? 1 : (g & 4) ? 2 : (g & 8) ? 3 : 4; }

// Per-class launch arguments.
template <typename T>
struct QArgs {
    typename C2<T>::t* amps;       // circuit c at amps + c * 2^n
    uint64_t ncirc;                // circuits in this wave
    uint64_t ntiles;               // tiles per circuit
    uint64_t circ0;                // global index of the wave's first circuit
    const uint32_t* circ_inst;     // global circuit -> instance
    const uint8_t* edges;          // (u, v) byte pairs of all instances
    const uint32_t* eoff;          // instance -> first edge
    const uint32_t* ne;            // instance -> edge count
    const uint64_t* nbr;           // instance -> NBR_STRIDE neighbour masks (bit w of entry v: edge (v, w))
    const T* rot;                  // [global circuit][nparam] (cos, sin) of Rx(2 beta) / Ry(theta) half-angles
    uint32_t nparam;
    const T* ph;                   // [global circuit][p][phs] (re, im) of exp(-i gamma (|E| - 2k))
    uint32_t p, phs;
    double* epart;                 // [wave circuit][ntiles]
    T amp0;                        // 2^(-n/2)
    typename C2<T>::t* lam;        // adjoint sweeps: lambda of circuit c at lam + c * 2^n
    double* gpart;                 // adjoint sweeps: [wave circuit][ntiles][gwidth] gradient partials
    uint32_t gwidth;               // adjoint sweeps: gradient entries per circuit (2p for QAOA, P for VQE)
};

// cut(x) for the register amplitudes of one thread, x = U | deposit(i), from the graph's
// neighbour masks N(v), for U with every slot bit 0:
//   cut(U)             = sum over vertices v with U_v = 1 of popc(N(v) & ~U)
//   flipping slot s    : delta_s = deg(s) - 2 popc(N(s) & U)   (slot neighbours count as 0)
//   slots s, t both 1  : their shared edge was counted twice by delta_s + delta_t, -2 each
// so cut(U | deposit(i)) = c0 + sum_{s in i} delta_s - 2 #(adjacent slot pairs in i).
constexpr uint32_t NBR_STRIDE = 32;   // batched graphs have at most 30 vertices

template <int RB>
struct CutNb {
    int c0;
    int delta[RB];
    uint32_t adj;      // bit s * RB + t (s < t): slots s and t adjacent
};

template <int RB>
__device__ __forceinline__ void cut_plan_nb(CutNb<RB>& cp, const uint64_t* __restrict__ nb, uint64_t U,
                                            const uint8_t* slot_global) {
    int c0 = 0;
    for (uint64_t m = U; m; m &= m - 1) c0 += __popcll(nb[__ffsll((long long)m) - 1] & ~U);
    cp.c0 = c0;
    cp.adj = 0;
#pragma unroll
    for (int s = 0; s < RB; ++s) {
        const uint64_t ns = nb[slot_global[s]];
        cp.delta[s] = __popcll(ns) - 2 * __popcll(ns & U);
#pragma unroll
        for (int t = s + 1; t < RB; ++t)
            if ((ns >> slot_global[t]) & 1ull) cp.adj |= 1u << (s * RB + t);
    }
}

template <int RB>
__device__ __forceinline__ int cut_nb(const CutNb<RB>& cp, int i) {   // i: a compile-time register index
    int c = cp.c0;
#pragma unroll
    for (int s = 0; s < RB; ++s)
        if ((i >> s) & 1) c += cp.delta[s];
#pragma unroll
    for (int s = 0; s < RB; ++s)
#pragma unroll
        for (int t = s + 1; t < RB; ++t)
            if (((i >> s) & 1) && ((i >> t) & 1)) c -= 2 * (int)((cp.adj >> (s * RB + t)) & 1u);
    return c;
}

// v * i^k (exact: a swap and sign changes)
template <typename V>
__device__ __forceinline__ V mul_ipow(V v, int k) {
    V r;
    switch (k & 3) {
        case 0: r = v; break;
        case 1: r.x = -v.y; r.y = v.x; break;
        case 2: r.x = -v.x; r.y = -v.y; break;
        default: r.x = v.y; r.y = -v.x; break;
    }
    return r;
}

template <typename V, typename T>
__device__ __forceinline__ V cmulv(V a, T br, T bi) {
    V r;
    r.x = a.x * br - a.y * bi;
    r.y = a.x * bi + a.y * br;
    return r;
}

// Rx(2 beta) on slot K: [[c, -i s], [-i s, c]]
template <int K, int NR, typename V, typename T>
__device__ __forceinline__ void op_rx(V* reg, T c, T s) {
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (i & (1 << K)) continue;
        const int j = i | (1 << K);
        V x = reg[i], y = reg[j];
        V o0, o1;
        o0.x = c * x.x + s * y.y;
        o0.y = c * x.y - s * y.x;
        o1.x = s * x.y + c * y.x;
        o1.y = c * y.y - s * x.x;
        reg[i] = o0;
        reg[j] = o1;
    }
}

template <int NR, typename V, typename T>
__device__ __forceinline__ void dispatch_rx(int k, V* reg, T c, T s) {
    switch (k) {
        case 0: op_rx<0, NR>(reg, c, s); break;
        case 1: op_rx<1, NR>(reg, c, s); break;
        case 2: op_rx<2, NR>(reg, c, s); break;
        case 3: if constexpr (NR > 8) op_rx<3, NR>(reg, c, s); break;
        case 4: if constexpr (NR > 16) op_rx<4, NR>(reg, c, s); break;
        default: break;
    }
}

// packed FP32x2 arithmetic: one instruction for both parts of a complex f32 value
__device__ __forceinline__ float2 pk_mul(float2 a, float2 b) {
    float2 r;
    asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 pk_fma(float2 a, float2 b, float2 c) {
    float2 r;
    asm("{.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rc, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}

// Ry(theta) on slot K: [[c, -s], [s, c]] with c = cos(theta/2), s = sin(theta/2)
template <int K, int NR, typename V, typename T>
__device__ __forceinline__ void op_ry(V* reg, T c, T s) {
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (i & (1 << K)) continue;
        const int j = i | (1 << K);
        V x = reg[i], y = reg[j];
        V o0, o1;
        if constexpr (std::is_same<T, float>::value) {   // c x - s y and s x + c y, both parts at once
            const float2 c2 = make_float2(c, c), s2 = make_float2(s, s), ms2 = make_float2(-s, -s);
            o0 = pk_fma(c2, x, pk_mul(ms2, y));
            o1 = pk_fma(s2, x, pk_mul(c2, y));
        } else {
            o0.x = c * x.x - s * y.x;
            o0.y = c * x.y - s * y.y;
            o1.x = s * x.x + c * y.x;
            o1.y = s * x.y + c * y.y;
        }
        reg[i] = o0;
        reg[j] = o1;
    }
}

template <int NR, typename V, typename T>
__device__ __forceinline__ void dispatch_ry(int k, V* reg, T c, T s) {
    switch (k) {
        case 0: op_ry<0, NR>(reg, c, s); break;
        case 1: op_ry<1, NR>(reg, c, s); break;
        case 2: op_ry<2, NR>(reg, c, s); break;
        case 3: if constexpr (NR > 8) op_ry<3, NR>(reg, c, s); break;
        case 4: if constexpr (NR > 16) op_ry<4, NR>(reg, c, s); break;
        default: break;
    }
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void bcp_async8(void* smem, const void* gmem) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void bcp_async16(void* smem, const void* gmem) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// Batched QAOA sweep over (circuit, tile) work items of one class.
template <typename T, int RB>
__global__ void __launch_bounds__(256, 2) k_batch_sweep(const SweepDesc d, const PhaseDesc* __restrict__ phases,
                                                      const SwOp* __restrict__ ops, QArgs<T> a) {
    using V = typename C2<T>::t;
    using VV = typename Vec16b<T>::t;
    constexpr int NR = 1 << RB;
    constexpr int EPV = Vec16b<T>::EPV;
    constexpr int VPT = NR / EPV;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* sm = reinterpret_cast<V*>(smem_raw);
    __shared__ double red[256];

    const uint32_t tid = threadIdx.x;
    const uint32_t T_ = blockDim.x;
    const uint64_t cmask = (1ull << d.c) - 1;
    uint64_t dep_tid = 0;
    {
        uint64_t x = (uint64_t)tid * EPV;
        dep_tid = x & cmask;
        for (uint32_t b = d.c; b < d.m; ++b)
            if ((x >> b) & 1ull) dep_tid |= 1ull << d.local_global[b];
    }
    // complex f32 programs use the layout of swz16 (retable_f16: every local bit has its own
    // bank pattern, warp lanes span the banks); complex f64 programs the row swizzle swzb
    constexpr bool F16L = std::is_same<T, float>::value;
    const uint32_t stid = F16L ? swz16(tid * EPV) : swzb<T>(tid * EPV);   // swz(e) = stid ^ sgj[j] (XOR-linear)
    const uint64_t nwork = a.ncirc * a.ntiles;
    const uint64_t nstate = 1ull << d.n;
    // the sweep's phase descriptors in shared memory, after the tile
    PhaseDesc* sph = reinterpret_cast<PhaseDesc*>(smem_raw + ((size_t)1 << d.m) * sizeof(V));
    {
        const uint32_t nw = (d.phase_end - d.phase_begin) * (uint32_t)(sizeof(PhaseDesc) / 16);
        const uint4* src = reinterpret_cast<const uint4*>(phases + d.phase_begin);
        for (uint32_t k = tid; k < nw; k += T_) reinterpret_cast<uint4*>(sph)[k] = src[k];
    }
    __syncthreads();

    for (uint64_t w = blockIdx.x; w < nwork; w += gridDim.x) {
        const uint64_t circ = w / a.ntiles, tile = w - circ * a.ntiles;
        const uint64_t gcirc = a.circ0 + circ;
        V* amps = a.amps + circ * nstate;
        const uint64_t* nb = nullptr;   // the instance's neighbour masks (cost phase and energy)
        if (a.circ_inst) nb = a.nbr + (size_t)a.circ_inst[gcirc] * NBR_STRIDE;
        uint64_t base = 0;
        for (uint32_t b = 0; b < d.nonlocal_count; ++b)
            if ((tile >> b) & 1ull) base |= 1ull << d.nonlocal[b];

        const bool init = (d.flags & (SWEEP_INIT_UNIFORM | SWEEP_INIT_ZERO)) != 0;
        if (!init) {
            // all of the tile's copies in flight at once (cp.async, element-granular for the swizzle)
#pragma unroll
            for (int j = 0; j < VPT; ++j) {
                const V* g = amps + (base | dep_tid | d.gj[j]);
                const uint32_t se = stid ^ d.sgj[j];
                if constexpr (EPV == 2) {
                    bcp_async8(sm + se, g);
                    bcp_async8(sm + (se ^ 1u), g + 1);
                } else {
                    bcp_async16(sm + se, g);
                }
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();

        double energy = 0.0;
        for (uint32_t p = d.phase_begin; p < d.phase_end; ++p) {
            const PhaseDesc& ph = sph[p - d.phase_begin];
            uint32_t ebase = 0;
            uint64_t U = base;
            for (uint32_t b = 0; b < ph.nt; ++b)
                if ((tid >> b) & 1u) {
                    ebase |= 1u << ph.tbit_local[b];
                    U |= 1ull << ph.tbit_global[b];
                }
            const uint32_t sb = F16L ? swz16(ebase) : swzb<T>(ebase);
            // register i sits at sb ^ (XOR of S[k] over the set bits k of i): visited in
            // Gray-code order, each address is one XOR from the previous one
            uint32_t S[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k) S[k] = ph.slut[1 << k];
            V reg[NR];
            if (init && p == d.phase_begin) {
                if (d.flags & SWEEP_INIT_UNIFORM) {
#pragma unroll
                    for (int i = 0; i < NR; ++i) { reg[i].x = a.amp0; reg[i].y = (T)0; }
                    if (d.flags & SWEEP_PHASE_IN) {   // S^n H^n |0>: amplitude i^popc(x)
                        const int pu = __popcll(U);
#pragma unroll
                        for (int i = 0; i < NR; ++i) reg[i] = mul_ipow(reg[i], pu + __popc(i));
                    }
                } else {   // |0...0>
#pragma unroll
                    for (int i = 0; i < NR; ++i) { reg[i].x = (i == 0 && U == 0) ? (T)1 : (T)0; reg[i].y = (T)0; }
                }
            } else {
                uint32_t ad = sb;
#pragma unroll
                for (int g = 0; g < NR; ++g) {
                    if (g) ad ^= S[gray_bit(g)];
                    reg[g ^ (g >> 1)] = sm[ad];
                }
            }
            for (uint32_t o = ph.op_begin; o < ph.op_end; ++o) {
                const SwOp op = ops[o];
                if (op.type == OP_RXP) {
                    const T* r = a.rot + ((size_t)gcirc * a.nparam + op.param) * 2;
                    dispatch_rx<NR>(op.k0, reg, r[0], r[1]);
                } else if (op.type == OP_RYP) {
                    const T* r = a.rot + ((size_t)gcirc * a.nparam + op.param) * 2;
                    dispatch_ry<NR>(op.k0, reg, r[0], r[1]);
                } else if (op.type == OP_CZ) {
                    const int k0 = op.k0, k1 = op.k1;
                    const int u0 = (int)((U >> op.q0) & 1ull), u1 = (int)((U >> op.q1) & 1ull);
#pragma unroll
                    for (int i = 0; i < NR; ++i) {
                        const int b0 = k0 >= 0 ? ((i >> k0) & 1) : u0;
                        const int b1 = k1 >= 0 ? ((i >> k1) & 1) : u1;
                        if (b0 & b1) { reg[i].x = -reg[i].x; reg[i].y = -reg[i].y; }
                    }
                } else if (op.type == OP_CPH) {
                    CutNb<RB> cp;
                    cut_plan_nb<RB>(cp, nb, U, ph.slot_global);
                    const T* tab = a.ph + ((size_t)gcirc * a.p + op.param) * a.phs * 2;
#pragma unroll
                    for (int i = 0; i < NR; ++i) {
                        const int c = cut_nb<RB>(cp, i);
                        reg[i] = cmulv(reg[i], tab[2 * c], tab[2 * c + 1]);
                    }
                }
            }
            if ((d.flags & SWEEP_PHASE_OUT) && p + 1 == d.phase_end) {   // S^dag on every qubit
                const int pu = __popcll(U);
#pragma unroll
                for (int i = 0; i < NR; ++i) reg[i] = mul_ipow(reg[i], -(pu + __popc(i)));
            }
            if ((d.flags & SWEEP_ENERGY) && p + 1 == d.phase_end) {
                CutNb<RB> cp;
                cut_plan_nb<RB>(cp, nb, U, ph.slot_global);
                T e = 0;   // this thread's 2^RB terms in the state's type, then FP64 across threads
#pragma unroll
                for (int i = 0; i < NR; ++i)
                    e += (reg[i].x * reg[i].x + reg[i].y * reg[i].y) * (T)cut_nb<RB>(cp, i);
                energy += (double)e;
            }
            {
                uint32_t ad = sb;
#pragma unroll
                for (int g = 0; g < NR; ++g) {
                    if (g) ad ^= S[gray_bit(g)];
                    sm[ad] = reg[g ^ (g >> 1)];
                }
            }
            __syncthreads();
        }

        if (d.flags & SWEEP_ENERGY) {
            // fixed-order sum over the block (any block size, also < 32 threads)
            red[tid] = energy;
            __syncthreads();
            if (tid == 0) {
                double r = 0.0;
                for (uint32_t k = 0; k < T_; ++k) r += red[k];
                a.epart[circ * a.ntiles + tile] = r;
            }
            __syncthreads();
        }

#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            const uint32_t se = stid ^ d.sgj[j];
            const uint64_t g = base | dep_tid | d.gj[j];
            VV v;
            if constexpr (EPV == 2) {
                float2 x = sm[se], y = sm[se ^ 1u];
                v = make_float4(x.x, x.y, y.x, y.y);
            } else {
                V x = sm[se];
                v = *reinterpret_cast<VV*>(&x);
            }
            __stcs(reinterpret_cast<VV*>(amps + g), v);
        }
        __syncthreads();
    }
}

// energies[circ0 + c] = sum over the circuit's tile partials (fixed order)
__global__ void k_energy_finalize(const double* __restrict__ epart, uint64_t ncirc, uint64_t ntiles, uint64_t circ0,
                                  double* __restrict__ energies) {
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncirc; c += (uint64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (uint64_t t = 0; t < ntiles; ++t) s += epart[c * ntiles + t];
        energies[circ0 + c] = s;
    }
}

// ---- exact gradients: one adjoint sweep pass per circuit ------------------
//
// With psi = the final state and lambda = C psi (C = diag(cut(x))), the
// derivative of E = <psi|C|psi> by a parameter theta of a gate exp(-i theta G)
// is 2 Im <lambda_k|G|psi_k>, both vectors taken at that gate and carried
// backwards by applying each gate's inverse to both.  Per QAOA layer l (in
// reverse): dE/dbeta_l = sum_q 2 Im <lambda|X_q|psi> (Rx(2 beta) =
// exp(-i beta X); X_q commutes with every Rx of the layer, so the term is
// taken when Rx_q is undone), then dE/dgamma_l = 2 Im <lambda|G|psi> with
// G = diag(|E| - 2 cut(x)) (the product of the layer's Rzz(2 gamma) is
// exp(-i gamma G)).  Each thread holds the same 2^RB indices of psi and
// lambda; a thread sums its (at most 16) products of one op in the state's type,
// the per-op partials are FP64, reduced per warp by shuffles (fixed order) into
// per-warp rows of shared memory, and per tile into gpart -- deterministic for a
// given launch shape.
template <int K, int NR, typename V>
__device__ __forceinline__ double im_x_overlap(const V* p, const V* l) {
    decltype(p[0].x) acc = 0;   // at most 16 products of one thread, in the state's type
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (i & (1 << K)) continue;
        const int j = i | (1 << K);
        // Im(conj(l_i) p_j + conj(l_j) p_i)
        acc += (l[i].x * p[j].y - l[i].y * p[j].x) + (l[j].x * p[i].y - l[j].y * p[i].x);
    }
    return (double)acc;
}

template <int NR, typename V>
__device__ __forceinline__ double dispatch_im_x(int k, const V* p, const V* l) {
    switch (k) {
        case 0: return im_x_overlap<0, NR>(p, l);
        case 1: return im_x_overlap<1, NR>(p, l);
        case 2: return im_x_overlap<2, NR>(p, l);
        case 3: if constexpr (NR > 8) return im_x_overlap<3, NR>(p, l); break;
        case 4: if constexpr (NR > 16) return im_x_overlap<4, NR>(p, l); break;
        default: break;
    }
    return 0.0;
}

// Im <lambda|Y_K|psi> over the register pairs: Y|0> = i|1>, Y|1> = -i|0>, so
// <lambda|Y psi> = sum_pairs i conj(l_j) p_i - i conj(l_i) p_j and its imaginary
// part is Re(conj(l_j) p_i) - Re(conj(l_i) p_j).
template <int K, int NR, typename V>
__device__ __forceinline__ double im_y_overlap(const V* p, const V* l) {
    decltype(p[0].x) acc = 0;   // at most 16 products of one thread, in the state's type
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (i & (1 << K)) continue;
        const int j = i | (1 << K);
        acc += (l[j].x * p[i].x + l[j].y * p[i].y) - (l[i].x * p[j].x + l[i].y * p[j].y);
    }
    return (double)acc;
}

template <int NR, typename V>
__device__ __forceinline__ double dispatch_im_y(int k, const V* p, const V* l) {
    switch (k) {
        case 0: return im_y_overlap<0, NR>(p, l);
        case 1: return im_y_overlap<1, NR>(p, l);
        case 2: return im_y_overlap<2, NR>(p, l);
        case 3: if constexpr (NR > 8) return im_y_overlap<3, NR>(p, l); break;
        case 4: if constexpr (NR > 16) return im_y_overlap<4, NR>(p, l); break;
        default: break;
    }
    return 0.0;
}

template <typename T, int RB>
__global__ void __launch_bounds__(512, 1) k_batch_adjoint(const SweepDesc d, const PhaseDesc* __restrict__ phases,
                                                        const SwOp* __restrict__ ops, QArgs<T> a) {
    using V = typename C2<T>::t;
    using VV = typename Vec16b<T>::t;
    constexpr int NR = 1 << RB;
    constexpr int EPV = Vec16b<T>::EPV;
    constexpr int VPT = NR / EPV;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t tile_elems = 1u << d.m;
    V* smp = reinterpret_cast<V*>(smem_raw);
    V* sml = smp + tile_elems;
    double* gw = reinterpret_cast<double*>(sml + tile_elems);   // [group][2p]

    const uint32_t tid = threadIdx.x;
    const uint32_t T_ = blockDim.x;
    const bool small = T_ < 32;                  // tiny blocks: one row per thread, no shuffles
    const uint32_t ngroup = small ? T_ : (T_ >> 5);
    const uint32_t grp = small ? tid : (tid >> 5);
    const uint32_t lane = tid & 31u;
    const uint32_t P2 = a.gwidth;
    const uint64_t cmask = (1ull << d.c) - 1;
    uint64_t dep_tid = 0;
    {
        uint64_t x = (uint64_t)tid * EPV;
        dep_tid = x & cmask;
        for (uint32_t b = d.c; b < d.m; ++b)
            if ((x >> b) & 1ull) dep_tid |= 1ull << d.local_global[b];
    }
    const uint32_t stid = swzb<T>(tid * EPV);
    const uint64_t nwork = a.ncirc * a.ntiles;
    const uint64_t nstate = 1ull << d.n;
    const bool initl = (d.flags & SWEEP_INIT_LAMBDA) != 0;   // QAOA only: lambda = C psi

    auto flush = [&](double v, uint32_t idx) {
        if (!small) {
            v = warp_sum_d(v);
            if (lane == 0) gw[grp * P2 + idx] += v;
        } else {
            gw[grp * P2 + idx] += v;
        }
    };

    for (uint64_t w = blockIdx.x; w < nwork; w += gridDim.x) {
        const uint64_t circ = w / a.ntiles, tile = w - circ * a.ntiles;
        const uint64_t gcirc = a.circ0 + circ;
        V* psi = a.amps + circ * nstate;
        V* lam = a.lam + circ * nstate;
        const uint64_t* nb = nullptr;   // the instance's neighbour masks
        uint32_t ne = 0;
        if (a.circ_inst) {
            const uint32_t inst = a.circ_inst[gcirc];
            nb = a.nbr + (size_t)inst * NBR_STRIDE;
            ne = a.ne[inst];
        }
        uint64_t base = 0;
        for (uint32_t b = 0; b < d.nonlocal_count; ++b)
            if ((tile >> b) & 1ull) base |= 1ull << d.nonlocal[b];
        for (uint32_t k = tid; k < ngroup * P2; k += T_) gw[k] = 0.0;

#pragma unroll 1
        for (int j0 = 0; j0 < VPT; j0 += 4) {
            VV v[4], u[4];
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
                const uint64_t g = base | dep_tid | d.gj[j0 + jj];
                v[jj] = __ldcs(reinterpret_cast<const VV*>(psi + g));
                if (!initl) u[jj] = __ldcs(reinterpret_cast<const VV*>(lam + g));
            }
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
                const uint32_t se = stid ^ d.sgj[j0 + jj];
                if constexpr (EPV == 2) {
                    smp[se] = make_float2(v[jj].x, v[jj].y);
                    smp[se ^ 1u] = make_float2(v[jj].z, v[jj].w);
                    if (!initl) {
                        sml[se] = make_float2(u[jj].x, u[jj].y);
                        sml[se ^ 1u] = make_float2(u[jj].z, u[jj].w);
                    }
                } else {
                    smp[se] = *reinterpret_cast<V*>(&v[jj]);
                    if (!initl) sml[se] = *reinterpret_cast<V*>(&u[jj]);
                }
            }
        }
        __syncthreads();

        for (uint32_t p = d.phase_begin; p < d.phase_end; ++p) {
            const PhaseDesc& ph = phases[p];
            uint32_t ebase = 0;
            uint64_t U = base;
            for (uint32_t b = 0; b < ph.nt; ++b)
                if ((tid >> b) & 1u) {
                    ebase |= 1u << ph.tbit_local[b];
                    U |= 1ull << ph.tbit_global[b];
                }
            const uint32_t sb = swzb<T>(ebase);
            // register i sits at sb ^ (XOR of S[k] over the set bits k of i): Gray-code order
            uint32_t S[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k) S[k] = ph.slut[1 << k];
            V rp[NR], rl[NR];
            {
                uint32_t ad = sb;
#pragma unroll
                for (int g = 0; g < NR; ++g) {
                    if (g) ad ^= S[gray_bit(g)];
                    rp[g ^ (g >> 1)] = smp[ad];
                }
            }
            if (initl && p == d.phase_begin) {
                CutNb<RB> cp;
                cut_plan_nb<RB>(cp, nb, U, ph.slot_global);
#pragma unroll
                for (int i = 0; i < NR; ++i) {
                    const T c = (T)cut_nb<RB>(cp, i);
                    rl[i].x = c * rp[i].x;
                    rl[i].y = c * rp[i].y;
                }
            } else {
                uint32_t ad = sb;
#pragma unroll
                for (int g = 0; g < NR; ++g) {
                    if (g) ad ^= S[gray_bit(g)];
                    rl[g ^ (g >> 1)] = sml[ad];
                }
            }
            for (uint32_t o = ph.op_begin; o < ph.op_end; ++o) {
                const SwOp op = ops[o];
                if (op.type == OP_RXP) {
                    const T* r = a.rot + ((size_t)gcirc * a.nparam + op.param) * 2;
                    flush(2.0 * dispatch_im_x<NR>(op.k0, rp, rl), a.p + op.param);
                    dispatch_rx<NR>(op.k0, rp, r[0], -r[1]);
                    dispatch_rx<NR>(op.k0, rl, r[0], -r[1]);
                } else if (op.type == OP_CPH) {
                    CutNb<RB> cp;
                    cut_plan_nb<RB>(cp, nb, U, ph.slot_global);
                    const T* tab = a.ph + ((size_t)gcirc * a.p + op.param) * a.phs * 2;
                    T acc = 0;   // this thread's 2^RB terms in the state's type
#pragma unroll
                    for (int i = 0; i < NR; ++i) {
                        const int c = cut_nb<RB>(cp, i);
                        const T gdiag = (T)((int)ne - 2 * c);
                        acc += gdiag * (rl[i].x * rp[i].y - rl[i].y * rp[i].x);
                        rp[i] = cmulv(rp[i], tab[2 * c], -tab[2 * c + 1]);
                        rl[i] = cmulv(rl[i], tab[2 * c], -tab[2 * c + 1]);
                    }
                    flush(2.0 * (double)acc, op.param);
                } else if (op.type == OP_RYP) {
                    // Ry(theta) = exp(-i theta Y / 2): dE/dtheta = Im <lambda|Y|psi>
                    const T* r = a.rot + ((size_t)gcirc * a.nparam + op.param) * 2;
                    flush(dispatch_im_y<NR>(op.k0, rp, rl), op.param);
                    dispatch_ry<NR>(op.k0, rp, r[0], -r[1]);
                    dispatch_ry<NR>(op.k0, rl, r[0], -r[1]);
                } else if (op.type == OP_CZ) {   // self-inverse
                    const int k0 = op.k0, k1 = op.k1;
                    const int u0 = (int)((U >> op.q0) & 1ull), u1 = (int)((U >> op.q1) & 1ull);
#pragma unroll
                    for (int i = 0; i < NR; ++i) {
                        const int b0 = k0 >= 0 ? ((i >> k0) & 1) : u0;
                        const int b1 = k1 >= 0 ? ((i >> k1) & 1) : u1;
                        if (b0 & b1) {
                            rp[i].x = -rp[i].x;
                            rp[i].y = -rp[i].y;
                            rl[i].x = -rl[i].x;
                            rl[i].y = -rl[i].y;
                        }
                    }
                }
            }
            {
                uint32_t ad = sb;
#pragma unroll
                for (int g = 0; g < NR; ++g) {
                    if (g) ad ^= S[gray_bit(g)];
                    smp[ad] = rp[g ^ (g >> 1)];
                    sml[ad] = rl[g ^ (g >> 1)];
                }
            }
            __syncthreads();
        }

        for (uint32_t k = tid; k < P2; k += T_) {
            double s = 0.0;
            for (uint32_t g = 0; g < ngroup; ++g) s += gw[g * P2 + k];
            a.gpart[(circ * a.ntiles + tile) * P2 + k] = s;
        }
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            const uint32_t se = stid ^ d.sgj[j];
            const uint64_t g = base | dep_tid | d.gj[j];
            VV v, u;
            if constexpr (EPV == 2) {
                float2 x = smp[se], y = smp[se ^ 1u];
                v = make_float4(x.x, x.y, y.x, y.y);
                x = sml[se];
                y = sml[se ^ 1u];
                u = make_float4(x.x, x.y, y.x, y.y);
            } else {
                V x = smp[se];
                v = *reinterpret_cast<VV*>(&x);
                x = sml[se];
                u = *reinterpret_cast<VV*>(&x);
            }
            __stcs(reinterpret_cast<VV*>(psi + g), v);
            __stcs(reinterpret_cast<VV*>(lam + g), u);
        }
        __syncthreads();
    }
}

// grad[(circ0 + c) * P2 + k] += sum over the circuit's tile partials (fixed order)
__global__ void k_grad_finalize(const double* __restrict__ gpart, uint64_t ncirc, uint64_t ntiles, uint32_t P2,
                                uint64_t circ0, double* __restrict__ grad) {
    const uint64_t total = ncirc * P2;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = w / P2;
        const uint32_t k = (uint32_t)(w - c * P2);
        double s = 0.0;
        for (uint64_t t = 0; t < ntiles; ++t) s += gpart[(c * ntiles + t) * P2 + k];
        grad[(circ0 + c) * P2 + k] += s;
    }
}

// per-circuit tables from the angles: Rx(2 beta) -> (cos beta, sin beta);
// cost phase exp(-i gamma (|E| - 2k)) for k = 0..|E|
template <typename T>
__global__ void k_qaoa_tables(const double* __restrict__ gammas, const double* __restrict__ betas,
                              const uint32_t* __restrict__ circ_inst, const uint32_t* __restrict__ ne, uint64_t ncirc,
                              uint32_t p, uint32_t phs, T* __restrict__ rx, T* __restrict__ ph) {
    const uint64_t total = ncirc * p;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = w / p;
        const double g = gammas[w], b = betas[w];
        double sb, cb;
        sincos(b, &sb, &cb);
        rx[2 * w] = (T)cb;
        rx[2 * w + 1] = (T)sb;
        const int E = (int)ne[circ_inst[c]];
        T* t = ph + w * phs * 2;
        for (int k = 0; k < (int)phs; ++k) {
            double sv, cv;
            sincos(g * (double)(E - 2 * k), &sv, &cv);
            t[2 * k] = (T)cv;
            t[2 * k + 1] = (T)(-sv);
        }
    }
}

// ---- sampling -------------------------------------------------------------

template <typename T>
__device__ __forceinline__ double pr(const typename C2<T>::t* a, uint64_t i) {
    auto x = a[i];
    double re = x.x, im = x.y;
    return __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
}

// level n-1 of every circuit's tree (tree of circuit c at tree + c * 2^n)
template <typename T>
__global__ void k_bleaf(const typename C2<T>::t* __restrict__ amps, uint32_t n, uint64_t ncirc, double* __restrict__ tree) {
    const uint64_t half = 1ull << (n - 1), per = 1ull << n;
    const uint64_t total = ncirc * half;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = w >> (n - 1), j = w & (half - 1);
        const typename C2<T>::t* a = amps + c * per;
        tree[c * per + (half - 1) + j] = __dadd_rn(pr<T>(a, j), pr<T>(a, j + half));
    }
}

__global__ void k_bfold(double* __restrict__ tree, uint32_t n, uint64_t ncirc, uint32_t k) {
    const uint64_t len = 1ull << k, per = 1ull << n;
    const uint64_t total = ncirc * len;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = w >> k, j = w & (len - 1);
        double* t = tree + c * per;
        const double* up = t + ((1ull << (k + 1)) - 1);
        t[(len - 1) + j] = __dadd_rn(up[j], up[j + len]);
    }
}

// one block per circuit: shots, cut of each, best (max cut, lowest shot)
template <typename T>
__global__ void k_bsample(const typename C2<T>::t* __restrict__ amps, const double* __restrict__ tree, uint32_t n,
                          uint64_t ncirc, uint64_t circ0, const uint32_t* __restrict__ circ_inst,
                          const uint64_t* __restrict__ user_of,
                          const uint8_t* __restrict__ edges_all, const uint32_t* __restrict__ eoff,
                          const uint32_t* __restrict__ nes, uint32_t shots, uint64_t base_seed,
                          uint64_t* __restrict__ best_bits, uint32_t* __restrict__ best_cut) {
    __shared__ unsigned long long sh_key[32];
    __shared__ uint64_t sh_bits[32];
    const uint64_t per = 1ull << n;
    for (uint64_t c = blockIdx.x; c < ncirc; c += gridDim.x) {
        const uint64_t gc = circ0 + c;
        const typename C2<T>::t* a = amps + c * per;
        const double* t = tree + c * per;
        const uint32_t inst = circ_inst[gc];
        const uint8_t* e = edges_all + 2 * (size_t)eoff[inst];
        const uint32_t ne = nes[inst];
        // key orders by (cut desc, shot asc): (cut << 32) | (0xffffffff - shot)
        unsigned long long best = 0;
        uint64_t bbits = 0;
        for (uint32_t s = threadIdx.x; s < shots; s += blockDim.x) {
            const uint64_t key = base_seed + (user_of[gc] << 32) + s;
            uint64_t prefix = 0;
            for (uint32_t q = 0; q < n; ++q) {
                double m0, m1;
                if (q + 1 == n) {
                    m0 = pr<T>(a, prefix);
                    m1 = pr<T>(a, prefix | (1ull << q));
                } else {
                    const double* L = t + ((1ull << (q + 1)) - 1);
                    m0 = L[prefix];
                    m1 = L[prefix | (1ull << q)];
                }
                const double p0 = m0 / __dadd_rn(m0, m1);
                const double u = rqd::uniform(key, 0, q);
                if (u >= p0) prefix |= 1ull << q;
            }
            uint32_t cut = 0;
            for (uint32_t k = 0; k < ne; ++k) cut += (uint32_t)(((prefix >> e[2 * k]) ^ (prefix >> e[2 * k + 1])) & 1ull);
            const unsigned long long kk = ((unsigned long long)cut << 32) | (0xffffffffull - s);
            if (kk > best || (best == 0 && s == threadIdx.x)) {
                best = kk;
                bbits = prefix;
            }
        }
        // block argmax of the key
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long ok = __shfl_down_sync(0xffffffffu, best, o);
            uint64_t ob = __shfl_down_sync(0xffffffffu, bbits, o);
            if (ok > best) { best = ok; bbits = ob; }
        }
        if ((threadIdx.x & 31) == 0) { sh_key[threadIdx.x >> 5] = best; sh_bits[threadIdx.x >> 5] = bbits; }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long b = sh_key[0];
            uint64_t bb = sh_bits[0];
            for (uint32_t wv = 1; wv < (blockDim.x >> 5); ++wv)
                if (sh_key[wv] > b) { b = sh_key[wv]; bb = sh_bits[wv]; }
            best_bits[gc] = bb;
            best_cut[gc] = (uint32_t)(b >> 32);
        }
        __syncthreads();
    }
}


// ---- batched VQE -------------------------------------------------------------

// Pauli strings sharing one X/Y pattern (same rules as rq_reduce.cu):
// x == 0: acc += s(i)|a_i|^2 over all i; x != 0: over pairs (i, i^x) with the
// top bit h of x clear, acc += s(i) * (odd ? Im : Re) of conj(a_{i^x}) a_i.
struct VGroup {
    uint64_t x;
    uint32_t h, t0, nt, pad;
};
struct VTerm {
    uint64_t pmask;
    uint32_t odd, pad;
    double factor;   // coeff * the ny / pairing factor
};

template <typename T>
__global__ void k_vqe_energy(const typename C2<T>::t* __restrict__ states, uint32_t n, uint64_t ncirc, uint64_t circ0,
                             const VGroup* __restrict__ groups, uint32_t ngroups, const VTerm* __restrict__ terms,
                             double* __restrict__ energies) {
    __shared__ double red[8][8];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint64_t N = 1ull << n;
    for (uint64_t c = blockIdx.x; c < ncirc; c += gridDim.x) {
        const typename C2<T>::t* a = states + c * N;
        double E = 0.0;
        for (uint32_t g = 0; g < ngroups; ++g) {
            const VGroup G = groups[g];
            uint64_t pm[8];
            uint32_t od[8];
            double acc[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                pm[k] = k < (int)G.nt ? terms[G.t0 + k].pmask : 0;
                od[k] = k < (int)G.nt ? terms[G.t0 + k].odd : 0;
                acc[k] = 0.0;
            }
            const uint64_t count = G.x ? N >> 1 : N;
            for (uint64_t q = threadIdx.x; q < count; q += blockDim.x) {
                uint64_t i;
                double re, im;
                if (G.x == 0) {
                    i = q;
                    const auto v = a[i];
                    const double vr = v.x, vi = v.y;
                    re = vr * vr + vi * vi;
                    im = 0.0;
                } else {
                    i = rqd::insert0(q, G.h);
                    const auto ai = a[i];
                    const auto aj = a[i ^ G.x];
                    const double air = ai.x, aii = ai.y, ajr = aj.x, aji = aj.y;
                    re = ajr * air + aji * aii;
                    im = ajr * aii - aji * air;
                }
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const double v = od[k] ? im : re;
                    acc[k] += (__popcll(i & pm[k]) & 1) ? -v : v;
                }
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                double v = warp_sum_d(acc[k]);
                if (lane == 0) red[warp][k] = v;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                for (uint32_t k = 0; k < G.nt; ++k) {
                    double sum = 0.0;
                    for (uint32_t w = 0; w < nw; ++w) sum += red[w][k];
                    E += terms[G.t0 + k].factor * sum;
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) energies[circ0 + c] = E;
    }
}


// One Pauli group of a tile pass: NT strings (NT = 8 for 5..8), per-warp sums
// into wsum.  Products of amplitudes in the state's precision, every product
// added to an FP64 accumulator; indices fit 32 bits (at most 30 qubits).
// need: 1 = only Re of conj(a_j) a_i is used, 2 = only Im, 3 = both.
// a group's pairs are split into this many work units, so that the warps of a CTA finish a
// partner tile together (groups alone are too few and too coarse to balance 16 warps)
constexpr uint32_t VQE_CHUNKS = 4;

template <typename T, int NT>
__device__ __forceinline__ void tile_group(const VGroup& G, const VTerm* __restrict__ terms,
                                           const typename C2<T>::t* own, const typename C2<T>::t* src, uint32_t r,
                                           uint32_t rp, uint32_t t, uint32_t M, double* wsum, uint32_t nterms,
                                           uint32_t lane, uint32_t warp, uint32_t chunk, uint32_t nchunk) {
    using V = typename C2<T>::t;
    const uint32_t L = 1u << M;
    uint32_t pm[NT];
    bool od[NT];
    double acc[NT];
    int need = 0;
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        pm[k] = k < (int)G.nt ? (uint32_t)terms[G.t0 + k].pmask : 0u;
        od[k] = k < (int)G.nt ? terms[G.t0 + k].odd != 0 : false;
        if (k < (int)G.nt) need |= od[k] ? 2 : 1;
        acc[k] = 0.0;
    }
    const uint32_t x = (uint32_t)G.x;
    const uint32_t xl = x & (L - 1);
    const uint32_t count = x == 0 ? L : L >> 1;
    // this call's share of the group's pairs: chunk `chunk` of `nchunk` equal parts
    const uint32_t qlo = (uint32_t)(((uint64_t)count * chunk) / nchunk), qhi = (uint32_t)(((uint64_t)count * (chunk + 1)) / nchunk);
    const uint32_t sel = r < rp ? 0u : (1u ^ ((xl >> (M - 1)) & 1u));
    const uint32_t rbase = r << M, pbase = rp << M;
    // one warp owns the group: its lanes walk all pairs, one warp reduction per group.  The
    // products are summed in T over 16 pairs of a lane, then added into the FP64 accumulators
    // (16 terms in f32 keep the partial within ~1e-6 relative).
    for (uint32_t q0 = qlo + lane; q0 < qhi; q0 += 32 * 16) {
        T part[NT];
#pragma unroll
        for (int k = 0; k < NT; ++k) part[k] = (T)0;
#pragma unroll 4
        for (uint32_t u = 0; u < 16; ++u) {
            const uint32_t q = q0 + 32 * u;
            if (q >= qhi) break;
            T re = 0, im = 0;
            uint32_t i;
            if (x == 0) {
                i = rbase | q;
                const V v = own[q];
                re = v.x * v.x + v.y * v.y;
            } else {
                V af, as;
                if (t == 0) {
                    const uint32_t e = (uint32_t)rqd::insert0(q, G.h);
                    i = rbase | e;
                    af = own[e];
                    as = own[e ^ xl];
                } else {
                    const uint32_t e = (uint32_t)rqd::insert0(q, M - 1) | (sel << (M - 1));
                    const uint32_t ep = e ^ xl;
                    const uint32_t im_ = rbase | e;
                    const V ao = own[e], ap = src[ep];
                    const bool first_is_mine = !((im_ >> G.h) & 1u);
                    i = first_is_mine ? im_ : (pbase | ep);
                    af = first_is_mine ? ao : ap;
                    as = first_is_mine ? ap : ao;
                }
                if (need & 1) re = as.x * af.x + as.y * af.y;
                if (need & 2) im = as.x * af.y - as.y * af.x;
            }
#pragma unroll
            for (int k = 0; k < NT; ++k) {
                const T v = od[k] ? im : re;
                part[k] += (__popc(i & pm[k]) & 1) ? -v : v;
            }
        }
#pragma unroll
        for (int k = 0; k < NT; ++k) acc[k] += (double)part[k];
    }
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        const double v = warp_sum_d(acc[k]);
        if (lane == 0 && k < (int)G.nt) wsum[warp * nterms + G.t0 + k] += v;
    }
}

// Tiled form: the state of a circuit is split into ntile tiles of 2^M
// amplitudes; the CTA of (circuit, tile r) keeps tile r in shared memory and
// loads every partner tile r ^ t once, evaluating all Pauli groups whose X/Y
// pattern has top part x >> M == t from on-chip memory.  Pairs inside tile r
// (t = 0) are all counted by that CTA; pairs between tiles lo < hi are split
// by bit M-1 of their element in tile lo (0: CTA lo, 1: CTA hi), so each pair
// is counted once.  Each group is walked by one warp (groups dealt round-robin
// to the warps), whose per-string sums land in shared memory; the CTA writes one
// partial per string, and k_vqe_finalize adds the tiles and the strings in a
// fixed order.
template <typename T>
__global__ void __launch_bounds__(512, 1) k_vqe_energy_tiles(const typename C2<T>::t* __restrict__ states, uint32_t n,
                                                             uint32_t M, uint64_t ncirc,
                                                             const VGroup* __restrict__ groups,
                                                             const uint32_t* __restrict__ gofs, uint32_t nterms,
                                                             const VTerm* __restrict__ terms,
                                                             double* __restrict__ part) {
    using V = typename C2<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint64_t L = 1ull << M;
    V* own = reinterpret_cast<V*>(smem_raw);
    V* par = own + L;
    double* wsum = reinterpret_cast<double*>(par + L);   // [warps][nterms]
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t ntile = 1u << (n - M);
    const uint64_t N = 1ull << n;
    const uint64_t nwork = ncirc * ntile;
    for (uint64_t w = blockIdx.x; w < nwork; w += gridDim.x) {
        const uint64_t c = w / ntile;
        const uint32_t r = (uint32_t)(w - c * ntile);
        const V* a = states + c * N;
        for (uint32_t k = threadIdx.x; k < nw * nterms; k += blockDim.x) wsum[k] = 0.0;
        for (uint64_t e = threadIdx.x; e < L; e += blockDim.x) own[e] = a[((uint64_t)r << M) | e];
        __syncthreads();
        for (uint32_t t = 0; t < ntile; ++t) {
            if (gofs[t] == gofs[t + 1]) continue;
            const uint32_t rp = r ^ t;
            const V* src = own;
            if (t) {
                for (uint64_t e = threadIdx.x; e < L; e += blockDim.x) par[e] = a[((uint64_t)rp << M) | e];
                __syncthreads();
                src = par;
            }
            // work units: each group's pairs in VQE_CHUNKS equal parts, dealt to the warps in turn
            // (a warp's partial sums of a term add up in its own row of wsum)
            const uint32_t nunits = (gofs[t + 1] - gofs[t]) * VQE_CHUNKS;
            for (uint32_t u = warp; u < nunits; u += nw) {
                const VGroup G = groups[gofs[t] + u / VQE_CHUNKS];
                const uint32_t ch = u % VQE_CHUNKS;
                switch (G.nt) {
                    case 1: tile_group<T, 1>(G, terms, own, src, r, rp, t, M, wsum, nterms, lane, warp, ch, VQE_CHUNKS); break;
                    case 2: tile_group<T, 2>(G, terms, own, src, r, rp, t, M, wsum, nterms, lane, warp, ch, VQE_CHUNKS); break;
                    case 3: tile_group<T, 3>(G, terms, own, src, r, rp, t, M, wsum, nterms, lane, warp, ch, VQE_CHUNKS); break;
                    case 4: tile_group<T, 4>(G, terms, own, src, r, rp, t, M, wsum, nterms, lane, warp, ch, VQE_CHUNKS); break;
                    default: tile_group<T, 8>(G, terms, own, src, r, rp, t, M, wsum, nterms, lane, warp, ch, VQE_CHUNKS); break;
                }
            }
            __syncthreads();
        }
        for (uint32_t k = threadIdx.x; k < nterms; k += blockDim.x) {
            double sum = 0.0;
            for (uint32_t wv = 0; wv < nw; ++wv) sum += wsum[wv * nterms + k];
            part[w * nterms + k] = sum;
        }
        __syncthreads();
    }
}

// energies[circ0 + c] = sum over strings (in order) of factor * sum over tiles
__global__ void k_vqe_finalize(const double* __restrict__ part, uint64_t ncirc, uint32_t ntile, uint32_t nterms,
                               const VTerm* __restrict__ terms, uint64_t circ0, double* __restrict__ energies) {
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncirc; c += (uint64_t)gridDim.x * blockDim.x) {
        double E = 0.0;
        for (uint32_t k = 0; k < nterms; ++k) {
            double s = 0.0;
            for (uint32_t r = 0; r < ntile; ++r) s += part[(c * ntile + r) * nterms + k];
            E += terms[k].factor * s;
        }
        energies[circ0 + c] = E;
    }
}

// (cos, sin) of theta/2 for every (circuit, parameter): circuit = set * V + v;
// v = 0 is the set's parameters, v = 1 + 2k / 2 + 2k shift parameter k by +pi/2 / -pi/2
template <typename T>
__global__ void k_vqe_rot(const double* __restrict__ params, uint64_t ncirc, uint32_t P, uint32_t V, T* __restrict__ rot) {
    const uint64_t total = ncirc * P;
    const double hp = 1.57079632679489661923;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = w / P;
        const uint32_t k = (uint32_t)(w - c * P);
        const uint64_t set = c / V;
        const uint32_t v = (uint32_t)(c - set * V);
        double th = params[set * P + k];
        if (v > 0 && (v - 1) / 2 == k) th += (v & 1) ? hp : -hp;
        double sn, cs;
        sincos(0.5 * th, &sn, &cs);
        rot[2 * w] = (T)cs;
        rot[2 * w + 1] = (T)sn;
    }
}

constexpr int TPB = 256;

}  // namespace

// One Hamiltonian string as the operator i^ny X^x Z^pm: (P psi)[i] = c_k (-1)^popc((i^x) & pm) psi[i ^ x]
// with c_k = coeff * i^ny (ny = number of Y factors); (cr, ci) = c_k.
struct HTerm {
    uint64_t x, pm;
    double cr, ci;
};

// lambda = H psi for every circuit of a wave (the start of the VQE adjoint pass).  One
// output amplitude per thread and grid-stride step; the strings are read in order by
// every thread (uniform loads), psi[i ^ x] from L2 (a warp's 32 indices map to one
// aligned 32-amplitude block), the sum over strings in FP64.
template <typename T>
__global__ void __launch_bounds__(256) k_vqe_apply_h(const typename C2<T>::t* __restrict__ psi,
                                                     typename C2<T>::t* __restrict__ lam, uint32_t n, uint64_t ncirc,
                                                     const HTerm* __restrict__ terms, uint32_t nterms) {
    using V = typename C2<T>::t;
    const uint64_t N = 1ull << n;
    const uint64_t total = ncirc * N;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = w >> n, i = w & (N - 1);
        const V* src = psi + c * N;
        double re = 0.0, im = 0.0;
        for (uint32_t k = 0; k < nterms; ++k) {
            const HTerm t = terms[k];
            const uint64_t j = i ^ t.x;
            const V v = src[j];
            const double sg = (__popcll(j & t.pm) & 1) ? -1.0 : 1.0;
            const double cr = sg * t.cr, ci = sg * t.ci;
            re += cr * (double)v.x - ci * (double)v.y;
            im += cr * (double)v.y + ci * (double)v.x;
        }
        V o;
        o.x = (T)re;
        o.y = (T)im;
        lam[w] = o;
    }
}

// ===========================================================================
// batch object
// ===========================================================================
// Device-time and algorithmic-work accounting of one batched run, per kind of kernel
// (0: forward sweeps, 1: read-out -- QAOA sampling / VQE energies, 2: adjoint passes):
// events bracket each group of launches on the batch's stream; the sums are read after the
// run's final synchronisation.  Work is algorithmic: HBM bytes of the sweeps (S written by
// an initialising sweep, 2S per other sweep and state), the sampling tree's bytes, or the
// energy pass's floating-point operations.
struct RunProfile {
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;      // per event pair
    size_t used = 0;            // events in use
    bool on = false;            // only the plain runs are profiled (not graph-captured steps)
    double work[3] = {0, 0, 0};
    double ms[3] = {0, 0, 0};
    int begin(cudaStream_t st) {
        if (!on) return -1;
        if (used + 2 > ev.size()) {
            for (int k = 0; k < 2; ++k) {
                cudaEvent_t e = nullptr;
                if (cudaEventCreate(&e) != cudaSuccess) return -1;
                ev.push_back(e);
            }
        }
        cudaEventRecord(ev[used], st);
        used += 2;
        return (int)used - 2;
    }
    void end(int at, cudaStream_t st, int k, double w) {
        if (at < 0) return;
        cudaEventRecord(ev[at + 1], st);
        kind.push_back(k);
        work[k] += w;
    }
    void start() {
        on = true;
        used = 0;
        kind.clear();
        for (int k = 0; k < 3; ++k) work[k] = ms[k] = 0.0;
    }
    void collect() {   // after the stream has been synchronised
        on = false;
        for (size_t i = 0; i < kind.size(); ++i) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]) == cudaSuccess) ms[kind[i]] += t;
        }
    }
    void release() {
        for (auto e : ev) cudaEventDestroy(e);
        ev.clear();
    }
};

// algorithmic HBM bytes of one circuit's sweeps
inline double sweep_bytes(const std::vector<SweepDesc>& descs, double state_bytes, double states = 1.0) {
    double b = 0.0;
    for (const auto& d : descs) {
        const bool init = d.flags & (SWEEP_INIT_UNIFORM | SWEEP_INIT_ZERO);
        b += states * (init ? state_bytes : 2.0 * state_bytes);
        if (d.flags & SWEEP_INIT_LAMBDA) b -= state_bytes;   // lambda is built, not loaded
    }
    return b;
}

// A run's kernels as one CUDA graph.  The first run of a shape (sizes, modes, seeds and
// every buffer address the kernels see) launches plainly and is the profiled one; the next
// run of the same shape captures the same launch sequence and launches the graph, and later
// runs replay it.  A replay issues exactly the captured kernels with the captured
// arguments, so its results are those of a plain run.  RUQU_NO_GRAPHS=1 or
// rq_*_batch_set_graphs(0) keeps every run plain.
struct RunGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> key;      // shape of the last plain run (after it ran)
    bool enabled = std::getenv("RUQU_NO_GRAPHS") == nullptr;
    bool replayed = false;          // the last run launched the graph
    uint64_t nodes = 0;             // kernels (graph nodes) of the captured run
    void drop() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
    }
    // enqueue() issues the run's work on st; key_now() gives the shape; ev0 is recorded right
    // before the work (plain or graph)
    template <class F, class K>
    int run(cudaStream_t st, cudaEvent_t ev0, RunProfile& prof, F enqueue, K key_now) {
        replayed = false;
        const std::vector<uint64_t> k0 = key_now();
        const bool same = enabled && !key.empty() && k0 == key;
        if (!same) drop();
        if (same && !exec) {
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed);
            const int crc = e == cudaSuccess ? enqueue() : RQ_ERR_CUDA;
            const cudaError_t e2 = e == cudaSuccess ? cudaStreamEndCapture(st, &g) : e;
            bool ok = crc == RQ_OK && e2 == cudaSuccess && g && key_now() == key;
            if (ok) {
                size_t nn = 0;
                cudaGraphGetNodes(g, nullptr, &nn);
                nodes = nn;
                ok = cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
            }
            if (g) cudaGraphDestroy(g);
            if (!ok) {   // capture did not work here: plain runs from now on
                exec = nullptr;
                enabled = false;
                cudaGetLastError();
            }
        }
        if (same && exec) {
            RQ_CUDA(cudaEventRecord(ev0, st));
            RQ_CUDA(cudaGraphLaunch(exec, st));
            replayed = true;
            return RQ_OK;
        }
        prof.start();
        RQ_CUDA(cudaEventRecord(ev0, st));
        const int rc = enqueue();
        if (rc != RQ_OK) {
            prof.on = false;
            key.clear();
            return rc;
        }
        key = key_now();
        return RQ_OK;
    }
    void collect(RunProfile& prof) {   // after the stream has been synchronised
        if (!replayed) prof.collect();
    }
};

struct QClass {
    uint32_t n = 0, m = 0, c = 0;
    std::vector<uint32_t> insts;            // instances of this size
    std::vector<SweepDesc> descs;
    unsigned char* prog = nullptr;          // phases | ops
    size_t off_ops = 0;
    size_t smem = 0;
    uint64_t ntiles = 0;
    // the adjoint program (exact gradients): both states' tiles in shared memory
    uint32_t am = 0;
    std::vector<SweepDesc> adescs;
    unsigned char* aprog = nullptr;
    size_t aoff_ops = 0;
    uint64_t antiles = 0;
};

struct rq_qaoa_batch {
    int device = 0;
    int32_t prec = RQ_F32;
    uint32_t ninst = 0, p = 0, phs = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<uint32_t> n_of, ne_of;
    std::vector<QClass> classes;
    // device copies
    uint8_t* d_edges = nullptr;
    uint32_t* d_eoff = nullptr;
    uint32_t* d_ne = nullptr;
    uint64_t* d_nbr = nullptr;             // [instance][NBR_STRIDE] neighbour masks
    // per-run buffers
    uint32_t* d_circ_inst = nullptr;       // global circuit -> instance (class-major order)
    uint64_t* d_user = nullptr;            // run position -> caller's circuit index
    size_t circ_cap = 0;
    double* d_ang = nullptr;               // gammas | betas in circuit order
    void* d_rx = nullptr;
    void* d_ph = nullptr;
    double* d_energy = nullptr;
    uint64_t* d_best_bits = nullptr;
    uint32_t* d_best_cut = nullptr;
    void* d_states = nullptr;              // wave buffer
    size_t states_cap = 0;                 // bytes
    double* d_epart = nullptr;
    size_t epart_cap = 0;                  // doubles
    double* d_tree = nullptr;
    size_t tree_cap = 0;                   // doubles
    void* d_lam = nullptr;                 // adjoint wave buffer (lambda)
    size_t lam_cap = 0;                    // bytes
    double* d_gpart = nullptr;             // adjoint per-tile gradient partials
    size_t gpart_cap = 0;                  // doubles
    double* d_grad = nullptr;              // [circuit][2p] gradients of the last adjoint run
    size_t grad_cap = 0;                   // doubles
    std::vector<uint64_t> order;           // run-order position -> user circuit index
    // last run: which wave holds which circuits (for rq_qaoa_batch_state)
    uint32_t last_nsets = 0;
    uint64_t last_wave_first = 0, last_wave_count = 0;
    uint32_t last_wave_n = 0;
    float last_ms = 0.f;
    RunProfile prof;
    RunGraph graph;                        // rq_qaoa_batch_run / _gradient
    size_t state_budget = (size_t)24 << 30;
    double conv_tol = 0.0;                 // optimizers: stop an instance when |E - E_prev| < conv_tol (0: off)
};

namespace {

size_t elem_size(int32_t prec) { return prec == RQ_F32 ? 8 : 16; }

// the most phases of one sweep (k_batch_sweep keeps a sweep's phase descriptors in shared memory)
size_t max_phases(const std::vector<SweepDesc>& descs) {
    size_t m = 0;
    for (const auto& d : descs) m = std::max<size_t>(m, d.phase_end - d.phase_begin);
    return m;
}

template <typename P>
int grow(P** ptr, size_t* cap, size_t need_elems) {
    if (*cap >= need_elems) return RQ_OK;
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc((void**)ptr, need_elems * sizeof(P));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return rq::fail(RQ_ERR_MEMORY_ALLOCATION,
                        "memory allocation failed: need " + std::to_string(need_elems * sizeof(P)) + " bytes");
    }
    *cap = need_elems;
    return RQ_OK;
}

template <typename P>
int dalloc_b(P** p, size_t n) {
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(1, n) * sizeof(P));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return rq::fail(RQ_ERR_MEMORY_ALLOCATION, "memory allocation failed: need " + std::to_string(n * sizeof(P)) + " bytes");
    }
    return RQ_OK;
}

int grow_bytes(void** ptr, size_t* cap, size_t bytes) {
    if (*cap >= bytes) return RQ_OK;
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return rq::fail(RQ_ERR_MEMORY_ALLOCATION, "memory allocation failed: need " + std::to_string(bytes) + " bytes");
    }
    *cap = bytes;
    return RQ_OK;
}

template <typename T>
int launch_class(rq_qaoa_batch* b, QClass& K, uint64_t ncirc, uint64_t circ0, void* states) {
    using V = typename C2<T>::t;
    const uint32_t rb = std::is_same<T, float>::value ? 5 : 4;
    constexpr int RBc = std::is_same<T, float>::value ? 5 : 4;
    QArgs<T> a{};
    a.amps = (V*)states;
    a.ncirc = ncirc;
    a.ntiles = K.ntiles;
    a.circ0 = circ0;
    a.circ_inst = b->d_circ_inst;
    a.edges = b->d_edges;
    a.eoff = b->d_eoff;
    a.ne = b->d_ne;
    a.nbr = b->d_nbr;
    a.rot = (const T*)b->d_rx;
    a.nparam = b->p;
    a.ph = (const T*)b->d_ph;
    a.p = b->p;
    a.phs = b->phs;
    a.epart = b->d_epart;
    a.amp0 = (T)std::sqrt(std::ldexp(1.0, -(int)K.n));
    const PhaseDesc* ph = reinterpret_cast<const PhaseDesc*>(K.prog);
    const SwOp* op = reinterpret_cast<const SwOp*>(K.prog + K.off_ops);
    auto kern = k_batch_sweep<T, RBc>;
    RQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K.smem));
    const unsigned threads = 1u << (K.m - rb);
    int per_sm = 0;
    RQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)threads, K.smem));
    if (per_sm < 1) return rq::fail(RQ_ERR_CUDA, "batched sweep kernel does not fit on an SM");
    const uint64_t work = ncirc * K.ntiles;
    const unsigned grid = (unsigned)std::min<uint64_t>(work, (uint64_t)rq::num_sms(b->device) * per_sm);
    for (const auto& d : K.descs) {
        kern<<<grid, threads, K.smem, b->stream>>>(d, ph, op, a);
        RQ_CUDA(cudaGetLastError());
    }
    k_energy_finalize<<<rq::grid_for(ncirc, TPB, rq::num_sms(b->device)), TPB, 0, b->stream>>>(
        b->d_epart, ncirc, K.ntiles, circ0, b->d_energy);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

// backward pass of one wave: psi (left by the forward sweeps) and lambda through the
// adjoint program; per-circuit gradients accumulate into d_grad (zeroed by the caller)
template <typename T>
int adjoint_class(rq_qaoa_batch* b, QClass& K, uint64_t ncirc, uint64_t circ0, void* states, void* lam) {
    using V = typename C2<T>::t;
    constexpr int RBc = std::is_same<T, float>::value ? 4 : 3;
    const uint32_t P2 = 2 * b->p;
    QArgs<T> a{};
    a.amps = (V*)states;
    a.lam = (V*)lam;
    a.ncirc = ncirc;
    a.ntiles = K.antiles;
    a.circ0 = circ0;
    a.circ_inst = b->d_circ_inst;
    a.edges = b->d_edges;
    a.eoff = b->d_eoff;
    a.ne = b->d_ne;
    a.nbr = b->d_nbr;
    a.rot = (const T*)b->d_rx;
    a.nparam = b->p;
    a.ph = (const T*)b->d_ph;
    a.p = b->p;
    a.phs = b->phs;
    a.gpart = b->d_gpart;
    a.gwidth = P2;
    const PhaseDesc* ph = reinterpret_cast<const PhaseDesc*>(K.aprog);
    const SwOp* op = reinterpret_cast<const SwOp*>(K.aprog + K.aoff_ops);
    auto kern = k_batch_adjoint<T, RBc>;
    const unsigned threads = 1u << (K.am - RBc);
    const unsigned ngroup = threads < 32 ? threads : threads / 32;
    const size_t smem = 2 * ((size_t)1 << K.am) * sizeof(V) + (size_t)ngroup * P2 * sizeof(double);
    RQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    RQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)threads, smem));
    if (per_sm < 1) return rq::fail(RQ_ERR_CUDA, "adjoint sweep kernel does not fit on an SM");
    const uint64_t work = ncirc * K.antiles;
    const unsigned grid = (unsigned)std::min<uint64_t>(work, (uint64_t)rq::num_sms(b->device) * per_sm);
    const int sms = rq::num_sms(b->device);
    for (const auto& d : K.adescs) {
        kern<<<grid, threads, smem, b->stream>>>(d, ph, op, a);
        RQ_CUDA(cudaGetLastError());
        k_grad_finalize<<<rq::grid_for(ncirc * P2, TPB, sms), TPB, 0, b->stream>>>(b->d_gpart, ncirc, K.antiles, P2,
                                                                                 circ0, b->d_grad);
        RQ_CUDA(cudaGetLastError());
    }
    return RQ_OK;
}

template <typename T>
int sample_class(rq_qaoa_batch* b, QClass& K, uint64_t ncirc, uint64_t circ0, void* states, uint32_t shots,
                 uint64_t seed) {
    using V = typename C2<T>::t;
    const uint32_t n = K.n;
    const uint64_t per = 1ull << n;
    // trees for as many circuits as the tree scratch allows
    const size_t tree_budget = (size_t)8 << 30;
    uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(ncirc, tree_budget / (per * sizeof(double))));
    RQ_TRY(grow(&b->d_tree, &b->tree_cap, chunk * per));
    const int sms = rq::num_sms(b->device);
    for (uint64_t c0 = 0; c0 < ncirc; c0 += chunk) {
        const uint64_t cn = std::min<uint64_t>(chunk, ncirc - c0);
        const V* a = (const V*)states + c0 * per;
        k_bleaf<T><<<rq::grid_for(cn * (per >> 1), TPB, sms), TPB, 0, b->stream>>>(a, n, cn, b->d_tree);
        RQ_CUDA(cudaGetLastError());
        for (int k = (int)n - 2; k >= 0; --k) {
            k_bfold<<<rq::grid_for(cn << k, TPB, sms), TPB, 0, b->stream>>>(b->d_tree, n, cn, (uint32_t)k);
            RQ_CUDA(cudaGetLastError());
        }
        const unsigned g = (unsigned)std::min<uint64_t>(cn, (uint64_t)sms * 8);
        k_bsample<T><<<g, 256, 0, b->stream>>>(a, b->d_tree, n, cn, circ0 + c0, b->d_circ_inst, b->d_user, b->d_edges, b->d_eoff,
                                               b->d_ne, shots, seed, b->d_best_bits, b->d_best_cut);
        RQ_CUDA(cudaGetLastError());
    }
    return RQ_OK;
}

}  // namespace

extern "C" {

int rq_qaoa_batch_create(uint32_t ninst, const uint32_t* num_nodes, const uint32_t* edge_offsets,
                         const uint32_t* edges, uint32_t p, int32_t precision, rq_qaoa_batch** out) {
    if (!out || (!num_nodes && ninst) || (!edge_offsets && ninst)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (precision != RQ_F32 && precision != RQ_F64)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "precision must be RQ_F32 or RQ_F64");
    if (p == 0 || p > 64) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "p must be in 1..64");
    const uint32_t rb = precision == RQ_F32 ? 5 : 4;
    const uint32_t mloc = precision == RQ_F32 ? 13 : 12;
    std::unique_ptr<rq_qaoa_batch> b(new rq_qaoa_batch());
    b->prec = precision;
    b->ninst = ninst;
    b->p = p;
    cudaGetDevice(&b->device);
    uint32_t maxe = 0;
    std::vector<uint8_t> ed;
    for (uint32_t k = 0; k < ninst; ++k) {
        uint32_t n = num_nodes[k];
        if (n < rb + 2 || n > 30)
            return rq::fail(RQ_ERR_INVALID_ARGUMENT, "batched QAOA takes " + std::to_string(rb + 2) +
                                                         "..30 qubits per graph, got " + std::to_string(n));
        uint32_t e0 = edge_offsets[k], e1 = edge_offsets[k + 1];
        if (e1 < e0) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "edge offsets must be non-decreasing");
        for (uint32_t e = e0; e < e1; ++e) {
            uint32_t u = edges[2 * e], v = edges[2 * e + 1];
            if (u >= n || v >= n)
                return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "edge endpoint out of range in graph " + std::to_string(k));
            if (u == v) return rq::fail(RQ_ERR_CIRCUIT, "circuit error: self-loop in graph " + std::to_string(k));
            for (uint32_t f = e0; f < e; ++f)
                if ((edges[2 * f] == u && edges[2 * f + 1] == v) || (edges[2 * f] == v && edges[2 * f + 1] == u))
                    return rq::fail(RQ_ERR_INVALID_ARGUMENT, "batched QAOA takes simple graphs: edge (" +
                                                                 std::to_string(u) + "," + std::to_string(v) +
                                                                 ") repeats in graph " + std::to_string(k));
            ed.push_back((uint8_t)u);
            ed.push_back((uint8_t)v);
        }
        b->n_of.push_back(n);
        b->ne_of.push_back(e1 - e0);
        maxe = std::max(maxe, e1 - e0);
    }
    b->phs = maxe + 1;
    // size classes and their programs
    std::map<uint32_t, std::vector<uint32_t>> by_n;
    for (uint32_t k = 0; k < ninst; ++k) by_n[b->n_of[k]].push_back(k);
    RQ_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    RQ_CUDA(cudaEventCreate(&b->ev0));
    RQ_CUDA(cudaEventCreate(&b->ev1));
    for (auto& kv : by_n) {
        QClass K;
        K.n = kv.first;
        K.insts = kv.second;
        K.m = std::min(K.n, mloc);
        K.c = std::min<uint32_t>(K.m, 5);
        K.ntiles = 1ull << (K.n - K.m);
        K.smem = ((size_t)1 << K.m) * elem_size(precision);
        // the circuit of qaoa.rs:125-153 after H^n: per layer the cost phase, then Rx on every
        // qubit, run as Ry between the phases S^n H^n |0> and a final S^dag n (SWEEP_PHASE_IN /
        // _OUT): a real rotation costs half the arithmetic of Rx
        std::vector<PGate> g;
        for (uint32_t l = 0; l < p; ++l) {
            PGate ph{};
            ph.type = OP_CPH;
            ph.q0 = 0;
            ph.q1 = 0;
            ph.param = (uint16_t)l;
            ph.span = (K.n >= 64) ? ~0ull : ((1ull << K.n) - 1);
            g.push_back(ph);
            for (uint32_t q = 0; q < K.n; ++q) {
                PGate rx{};
                rx.type = OP_RYP;
                rx.q0 = q;
                rx.param = (uint16_t)l;
                g.push_back(rx);
            }
        }
        auto sweeps = plan_sweeps(g, K.n, K.m, K.c);
        std::vector<PhaseDesc> phases;
        std::vector<SwOp> ops;
        std::vector<double> mats;
        build_program(sweeps, K.n, K.m, K.c, rb, precision == RQ_F32 ? 2 : 1, K.descs, phases, ops, mats);
        if (precision == RQ_F32) retable_f16(K.descs, phases, rb);   // the conflict-free layout (k_batch_sweep<float>)
        K.smem += max_phases(K.descs) * sizeof(PhaseDesc);   // the phase descriptors after the tile
        K.descs.front().flags |= SWEEP_INIT_UNIFORM | SWEEP_PHASE_IN;
        K.descs.back().flags |= SWEEP_ENERGY | SWEEP_PHASE_OUT;
        K.off_ops = (phases.size() * sizeof(PhaseDesc) + 255) & ~size_t(255);
        size_t total = K.off_ops + ops.size() * sizeof(SwOp);
        std::vector<unsigned char> host(total);
        std::memcpy(host.data(), phases.data(), phases.size() * sizeof(PhaseDesc));
        std::memcpy(host.data() + K.off_ops, ops.data(), ops.size() * sizeof(SwOp));
        RQ_CUDA(cudaMalloc((void**)&K.prog, total));
        RQ_CUDA(cudaMemcpy(K.prog, host.data(), total, cudaMemcpyHostToDevice));
        {
            // adjoint: per layer in reverse, Rx^-1 on every qubit, then the inverse cost phase
            const uint32_t arb = precision == RQ_F32 ? 4 : 3;
            K.am = std::min(K.n, mloc);
            K.antiles = 1ull << (K.n - K.am);
            const uint32_t ac = std::min<uint32_t>(K.am, 5);
            std::vector<PGate> ga;
            for (uint32_t l = p; l-- > 0;) {
                for (uint32_t q = 0; q < K.n; ++q) {
                    PGate rx{};
                    rx.type = OP_RXP;
                    rx.q0 = q;
                    rx.param = (uint16_t)l;
                    ga.push_back(rx);
                }
                PGate ph{};
                ph.type = OP_CPH;
                ph.param = (uint16_t)l;
                ph.span = (K.n >= 64) ? ~0ull : ((1ull << K.n) - 1);
                ga.push_back(ph);
            }
            auto asw = plan_sweeps(ga, K.n, K.am, ac);
            std::vector<PhaseDesc> aph;
            std::vector<SwOp> aops;
            std::vector<double> amats;
            build_program(asw, K.n, K.am, ac, arb, precision == RQ_F32 ? 2 : 1, K.adescs, aph, aops, amats);
            K.adescs.front().flags |= SWEEP_INIT_LAMBDA;
            K.aoff_ops = (aph.size() * sizeof(PhaseDesc) + 255) & ~size_t(255);
            const size_t atotal = K.aoff_ops + aops.size() * sizeof(SwOp);
            std::vector<unsigned char> ah(atotal);
            std::memcpy(ah.data(), aph.data(), aph.size() * sizeof(PhaseDesc));
            std::memcpy(ah.data() + K.aoff_ops, aops.data(), aops.size() * sizeof(SwOp));
            RQ_CUDA(cudaMalloc((void**)&K.aprog, atotal));
            RQ_CUDA(cudaMemcpy(K.aprog, ah.data(), atotal, cudaMemcpyHostToDevice));
        }
        b->classes.push_back(std::move(K));
    }
    // graph data
    if (ed.empty()) ed.push_back(0);
    RQ_CUDA(cudaMalloc((void**)&b->d_edges, ed.size()));
    RQ_CUDA(cudaMemcpy(b->d_edges, ed.data(), ed.size(), cudaMemcpyHostToDevice));
    std::vector<uint32_t> eoff(ninst + 1, 0);
    for (uint32_t k = 0; k < ninst; ++k) eoff[k + 1] = eoff[k] + b->ne_of[k];
    RQ_CUDA(cudaMalloc((void**)&b->d_eoff, (ninst + 1) * sizeof(uint32_t)));
    RQ_CUDA(cudaMemcpy(b->d_eoff, eoff.data(), (ninst + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice));
    RQ_CUDA(cudaMalloc((void**)&b->d_ne, std::max<uint32_t>(1, ninst) * sizeof(uint32_t)));
    if (ninst) RQ_CUDA(cudaMemcpy(b->d_ne, b->ne_of.data(), ninst * sizeof(uint32_t), cudaMemcpyHostToDevice));
    std::vector<uint64_t> nbr((size_t)std::max<uint32_t>(1, ninst) * NBR_STRIDE, 0);
    for (uint32_t k = 0; k < ninst; ++k)
        for (uint32_t e = eoff[k]; e < eoff[k + 1]; ++e) {
            const uint32_t u = ed[2 * (size_t)e], v = ed[2 * (size_t)e + 1];
            nbr[(size_t)k * NBR_STRIDE + u] |= 1ull << v;
            nbr[(size_t)k * NBR_STRIDE + v] |= 1ull << u;
        }
    RQ_CUDA(cudaMalloc((void**)&b->d_nbr, nbr.size() * sizeof(uint64_t)));
    RQ_CUDA(cudaMemcpy(b->d_nbr, nbr.data(), nbr.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
    // the copies above (from pageable memory) may return before their DMA lands, and the
    // batch's stream is not ordered after them: wait here, once, before any run
    RQ_CUDA(cudaDeviceSynchronize());
    *out = b.release();
    return RQ_OK;
}

int rq_qaoa_batch_destroy(rq_qaoa_batch* b) {
    if (!b) return RQ_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto& K : b->classes) {
        if (K.prog) cudaFree(K.prog);
        if (K.aprog) cudaFree(K.aprog);
    }
    void* ptrs[] = {b->d_edges, b->d_eoff, b->d_ne, b->d_nbr, b->d_circ_inst, b->d_user, b->d_ang, b->d_rx, b->d_ph, b->d_energy,
                    b->d_best_bits, b->d_best_cut, b->d_states, b->d_epart, b->d_tree, b->d_lam, b->d_gpart,
                    b->d_grad};
    for (void* q : ptrs) if (q) cudaFree(q);
    b->graph.drop();
    b->prof.release();
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return RQ_OK;
}

}  // extern "C"

namespace {

// Run order of circuits: class-major, then instance, then parameter set.
// Fills order / circ_inst, grows the per-run buffers, and (when gammas is not
// null) uploads the angles in run order.
int qaoa_prepare(rq_qaoa_batch* b, uint32_t nsets, const double* gammas, const double* betas) {
    const uint64_t ncirc = (uint64_t)b->ninst * nsets;
    const uint32_t p = b->p;
    b->order.clear();
    std::vector<uint32_t> circ_inst;
    std::vector<double> ang(gammas ? 2 * ncirc * p : 0);
    for (auto& K : b->classes)
        for (uint32_t inst : K.insts)
            for (uint32_t s = 0; s < nsets; ++s) {
                const uint64_t user = (uint64_t)inst * nsets + s;
                const uint64_t pos = b->order.size();
                b->order.push_back(user);
                circ_inst.push_back(inst);
                if (gammas)
                    for (uint32_t l = 0; l < p; ++l) {
                        ang[pos * p + l] = gammas[user * p + l];
                        ang[ncirc * p + pos * p + l] = betas[user * p + l];
                    }
            }
    size_t cap_ci = b->circ_cap;
    RQ_TRY(grow(&b->d_circ_inst, &cap_ci, ncirc));
    size_t cap_u = b->circ_cap;
    RQ_TRY(grow(&b->d_user, &cap_u, ncirc));
    size_t cap_a = b->circ_cap;
    RQ_TRY(grow(&b->d_ang, &cap_a, 2 * ncirc * p));
    size_t es = b->prec == RQ_F32 ? sizeof(float) : sizeof(double);
    size_t cap_rx = b->circ_cap ? b->circ_cap * p * 2 * es : 0;
    RQ_TRY(grow_bytes(&b->d_rx, &cap_rx, ncirc * p * 2 * es));
    size_t cap_ph = b->circ_cap ? b->circ_cap * p * b->phs * 2 * es : 0;
    RQ_TRY(grow_bytes(&b->d_ph, &cap_ph, ncirc * p * b->phs * 2 * es));
    size_t cap_e = b->circ_cap;
    RQ_TRY(grow(&b->d_energy, &cap_e, ncirc));
    size_t cap_bb = b->circ_cap;
    RQ_TRY(grow(&b->d_best_bits, &cap_bb, ncirc));
    size_t cap_bc = b->circ_cap;
    RQ_TRY(grow(&b->d_best_cut, &cap_bc, ncirc));
    b->circ_cap = std::max<size_t>(b->circ_cap, ncirc);
    RQ_CUDA(cudaMemcpyAsync(b->d_circ_inst, circ_inst.data(), ncirc * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
    RQ_CUDA(cudaMemcpyAsync(b->d_user, b->order.data(), ncirc * sizeof(uint64_t), cudaMemcpyHostToDevice, b->stream));
    if (gammas)
        RQ_CUDA(cudaMemcpyAsync(b->d_ang, ang.data(), ang.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    // the pageable sources must outlive the copies
    RQ_CUDA(cudaStreamSynchronize(b->stream));
    return RQ_OK;
}

// What a captured run depends on besides the uploaded angles: the run kind, sizes, seed and
// every buffer its kernels read or write.
std::vector<uint64_t> qaoa_shape(const rq_qaoa_batch* b, uint64_t kind, uint64_t nsets, uint64_t shots, uint64_t seed) {
    auto a = [](const void* p) { return (uint64_t)(uintptr_t)p; };
    return {kind, nsets, shots, seed, b->ninst, a(b->d_circ_inst), a(b->d_ang), a(b->d_rx), a(b->d_ph),
            a(b->d_energy), a(b->d_best_bits), a(b->d_best_cut), a(b->d_states), a(b->d_epart), a(b->d_tree),
            a(b->d_lam), a(b->d_gpart), a(b->d_grad), (uint64_t)b->state_budget};
}

// tables + every class's sweeps (+ shots) for the angles in d_ang; energies land in d_energy (run order).
// per_class (optional) gives how many instances of each size class the run holds, when the run is a
// compacted subset (the optimizer's still-active instances); d_circ_inst then lists only those.
// With adjoint set, every wave also runs the backward pass and d_grad receives the
// exact gradients ([run position][2p]: gammas, then betas).
int qaoa_launch(rq_qaoa_batch* b, uint32_t nsets, uint32_t shots, uint64_t base_seed,
                const std::vector<uint64_t>* per_class = nullptr, bool adjoint = false) {
    uint64_t nrun = 0;
    for (size_t k = 0; k < b->classes.size(); ++k) nrun += per_class ? (*per_class)[k] : b->classes[k].insts.size();
    const uint64_t ncirc = nrun * nsets;
    const uint32_t p = b->p;
    const int sms = rq::num_sms(b->device);
    if (b->prec == RQ_F32)
        k_qaoa_tables<float><<<rq::grid_for(ncirc * p, TPB, sms), TPB, 0, b->stream>>>(
            b->d_ang, b->d_ang + ncirc * p, b->d_circ_inst, b->d_ne, ncirc, p, b->phs, (float*)b->d_rx, (float*)b->d_ph);
    else
        k_qaoa_tables<double><<<rq::grid_for(ncirc * p, TPB, sms), TPB, 0, b->stream>>>(
            b->d_ang, b->d_ang + ncirc * p, b->d_circ_inst, b->d_ne, ncirc, p, b->phs, (double*)b->d_rx, (double*)b->d_ph);
    RQ_CUDA(cudaGetLastError());
    const uint32_t P2 = 2 * p;
    if (adjoint) {
        RQ_TRY(grow(&b->d_grad, &b->grad_cap, std::max<uint64_t>(1, ncirc) * P2));
        RQ_CUDA(cudaMemsetAsync(b->d_grad, 0, ncirc * P2 * sizeof(double), b->stream));
    }
    uint64_t pos = 0;
    for (size_t ki = 0; ki < b->classes.size(); ++ki) {
        auto& K = b->classes[ki];
        const uint64_t kc = (per_class ? (*per_class)[ki] : (uint64_t)K.insts.size()) * nsets;
        if (kc == 0) continue;
        const size_t state_bytes = ((size_t)1 << K.n) * elem_size(b->prec);
        const size_t per_circ = adjoint ? 2 * state_bytes : state_bytes;
        const uint64_t wave = std::max<uint64_t>(1, std::min<uint64_t>(kc, b->state_budget / per_circ));
        RQ_TRY(grow_bytes(&b->d_states, &b->states_cap, wave * state_bytes));
        RQ_TRY(grow(&b->d_epart, &b->epart_cap, wave * K.ntiles));
        if (adjoint) {
            RQ_TRY(grow_bytes(&b->d_lam, &b->lam_cap, wave * state_bytes));
            RQ_TRY(grow(&b->d_gpart, &b->gpart_cap, wave * K.antiles * P2));
        }
        for (uint64_t w0 = 0; w0 < kc; w0 += wave) {
            const uint64_t wn = std::min<uint64_t>(wave, kc - w0);
            const double sb = (double)state_bytes;
            int ev = b->prof.begin(b->stream);
            if (b->prec == RQ_F32) RQ_TRY(launch_class<float>(b, K, wn, pos + w0, b->d_states));
            else RQ_TRY(launch_class<double>(b, K, wn, pos + w0, b->d_states));
            b->prof.end(ev, b->stream, 0, (double)wn * sweep_bytes(K.descs, sb));
            if (shots) {
                ev = b->prof.begin(b->stream);
                if (b->prec == RQ_F32) RQ_TRY(sample_class<float>(b, K, wn, pos + w0, b->d_states, shots, base_seed));
                else RQ_TRY(sample_class<double>(b, K, wn, pos + w0, b->d_states, shots, base_seed));
                // the tree's leaf level reads the state and writes 2^n doubles; the folds read and
                // write the levels above once more (the walks touch n entries per shot)
                b->prof.end(ev, b->stream, 1, (double)wn * (sb + 2.0 * (double)((size_t)1 << K.n) * 8.0));
            }
            if (adjoint) {
                ev = b->prof.begin(b->stream);
                if (b->prec == RQ_F32) RQ_TRY(adjoint_class<float>(b, K, wn, pos + w0, b->d_states, b->d_lam));
                else RQ_TRY(adjoint_class<double>(b, K, wn, pos + w0, b->d_states, b->d_lam));
                b->prof.end(ev, b->stream, 2, (double)wn * sweep_bytes(K.adescs, sb, 2.0));
            }
            b->last_wave_first = pos + w0;
            b->last_wave_count = adjoint ? 0 : wn;   // the backward pass overwrites the final states
            b->last_wave_n = K.n;
        }
        pos += kc;
    }
    return RQ_OK;
}

// parameter sets of one optimizer step: set 0 = theta, set 1+2k / 2+2k = theta_k +- pi/2
// (the shift rule of run_qaoa, qaoa.rs:275-297); theta = (gamma_1..p, beta_1..p) per instance
// act lists the run-order instances still optimising; slot a of the run holds instance act[a].
__global__ void k_qaoa_shift(const double* __restrict__ theta, const uint32_t* __restrict__ act, uint32_t nact,
                             uint32_t p, uint32_t nsets, double* __restrict__ ang) {
    const uint64_t ncirc = (uint64_t)nact * nsets;
    const uint64_t total = ncirc * p;
    const double hp = 1.57079632679489661923;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = w / p;
        const uint32_t l = (uint32_t)(w - c * p);
        const uint64_t a = c / nsets;
        const uint32_t s = (uint32_t)(c - a * nsets);
        const uint64_t i = act[a];
        double g = theta[i * 2 * p + l], b = theta[i * 2 * p + p + l];
        if (s > 0) {
            const uint32_t k = (s - 1) / 2;
            const double d = (s & 1) ? hp : -hp;
            if (k == l) g += d;
            if (k == p + l) b += d;
        }
        ang[w] = g;
        ang[ncirc * p + w] = b;
    }
}

// one Adam step (gradient ascent on the expected cut) per instance, FP64 on the device;
// frozen once the target is met.  done[i] = 1 + the step at which the target was met.
// one preconditioned ascent step per instance: theta += alpha * P grad with the instance's
// 2p x 2p preconditioner P (a learned -H^-1); alpha halves whenever the energy fell since the
// previous step.  Frozen once the target is met, as the Adam step.
__global__ void k_qaoa_precond(const double* __restrict__ energy, const uint32_t* __restrict__ act, uint32_t nact,
                               uint32_t p, double* __restrict__ theta, const double* __restrict__ pre,
                               double* __restrict__ alpha, double* __restrict__ eprev,
                               const double* __restrict__ target, double rtol, uint32_t* __restrict__ done,
                               double* __restrict__ elast, int final_eval, const double* __restrict__ grad,
                               const uint32_t* __restrict__ step_dev, double conv) {
    const uint32_t step = *step_dev;
    const uint32_t P2 = 2 * p;
    for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < nact; a += gridDim.x * blockDim.x) {
        const uint32_t i = act[a];
        if (done[i]) continue;
        const double e = energy[a];
        elast[i] = e;
        if (target && e >= target[i] * (1.0 - rtol)) {
            done[i] = step + 1;
            continue;
        }
        if (conv > 0.0 && fabs(e - eprev[i]) < conv) {   // run_qaoa's convergence rule (qaoa.rs:266-269)
            done[i] = step + 1;
            continue;
        }
        if (final_eval) continue;
        if (e < eprev[i]) alpha[i] *= 0.5;
        eprev[i] = e;
        const double* g = grad + (uint64_t)a * P2;
        const double* P = pre + (uint64_t)i * P2 * P2;
        double d[128];
        for (uint32_t r = 0; r < P2; ++r) {
            double s = 0.0;
            for (uint32_t k = 0; k < P2; ++k) s += P[r * P2 + k] * g[k];
            d[r] = s;
        }
        for (uint32_t r = 0; r < P2; ++r) theta[(uint64_t)i * P2 + r] += alpha[i] * d[r];
    }
}

__global__ void k_step_inc(uint32_t* __restrict__ step) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *step += 1;
}

__global__ void k_qaoa_adam(const double* __restrict__ energy, const uint32_t* __restrict__ act, uint32_t nact,
                            uint32_t p, uint32_t nsets, double* __restrict__ theta, double* __restrict__ m,
                            double* __restrict__ v, double lr, uint32_t step, const double* __restrict__ target,
                            double rtol, uint32_t* __restrict__ done, double* __restrict__ elast, int final_eval,
                            const double* __restrict__ grad, const uint32_t* __restrict__ step_dev,
                            double* __restrict__ eprev, double conv) {
    if (step_dev) step = *step_dev;   // graph replays: the step counter lives on the device
    for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < nact; a += gridDim.x * blockDim.x) {
        const uint32_t i = act[a];
        if (done[i]) continue;
        const double* e = energy + (uint64_t)a * nsets;
        elast[i] = e[0];
        if (target && e[0] >= target[i] * (1.0 - rtol)) {
            done[i] = step + 1;
            continue;
        }
        if (conv > 0.0 && fabs(e[0] - eprev[i]) < conv) {   // run_qaoa's convergence rule (qaoa.rs:266-269)
            done[i] = step + 1;
            continue;
        }
        eprev[i] = e[0];
        if (final_eval) continue;
        const double b1 = 0.9, b2 = 0.999, eps = 1e-8;
        const double c1 = 1.0 - pow(b1, (double)(step + 1)), c2 = 1.0 - pow(b2, (double)(step + 1));
        for (uint32_t k = 0; k < 2 * p; ++k) {
            // exact (adjoint) gradient when given, else the shift rule of qaoa.rs:275-297
            const double g = grad ? grad[(uint64_t)a * 2 * p + k] : (e[1 + 2 * k] - e[2 + 2 * k]) / 2.0;
            const uint64_t j = (uint64_t)i * 2 * p + k;
            const double mm = b1 * m[j] + (1.0 - b1) * g;
            const double vv = b2 * v[j] + (1.0 - b2) * g * g;
            m[j] = mm;
            v[j] = vv;
            theta[j] += lr * (mm / c1) / (sqrt(vv / c2) + eps);
        }
    }
}

}  // namespace

extern "C" {

int rq_qaoa_batch_run(rq_qaoa_batch* b, uint32_t nsets, const double* gammas, const double* betas, double* energies,
                      uint32_t shots, uint64_t base_seed, uint64_t* best_bits, uint32_t* best_cut) {
    if (!b || !gammas || !betas || !energies) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (shots && (!best_bits || !best_cut)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null shot outputs");
    if (nsets == 0) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "nsets must be >= 1");
    RQ_CUDA(cudaSetDevice(b->device));
    const uint64_t ncirc = (uint64_t)b->ninst * nsets;
    RQ_TRY(qaoa_prepare(b, nsets, gammas, betas));
    RQ_TRY(b->graph.run(
        b->stream, b->ev0, b->prof, [&]() { return qaoa_launch(b, nsets, shots, base_seed); },
        [&]() { return qaoa_shape(b, 0, nsets, shots, base_seed); }));
    RQ_CUDA(cudaEventRecord(b->ev1, b->stream));
    std::vector<double> e(ncirc);
    RQ_CUDA(cudaMemcpyAsync(e.data(), b->d_energy, ncirc * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    std::vector<uint64_t> bb;
    std::vector<uint32_t> bc;
    if (shots) {
        bb.resize(ncirc);
        bc.resize(ncirc);
        RQ_CUDA(cudaMemcpyAsync(bb.data(), b->d_best_bits, ncirc * sizeof(uint64_t), cudaMemcpyDeviceToHost, b->stream));
        RQ_CUDA(cudaMemcpyAsync(bc.data(), b->d_best_cut, ncirc * sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream));
    }
    RQ_CUDA(cudaStreamSynchronize(b->stream));
    RQ_CUDA(cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
    b->graph.collect(b->prof);
    for (uint64_t k = 0; k < ncirc; ++k) {
        const uint64_t user = b->order[k];
        energies[user] = e[k];
        if (shots) {
            best_bits[user] = bb[k];
            best_cut[user] = bc[k];
        }
    }
    b->last_nsets = nsets;
    return RQ_OK;
}

int rq_qaoa_batch_gradient(rq_qaoa_batch* b, const double* gammas, const double* betas, double* energies,
                           double* gradients) {
    if (!b || !gammas || !betas || !energies || !gradients) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_CUDA(cudaSetDevice(b->device));
    const uint32_t p = b->p, P2 = 2 * p, ninst = b->ninst;
    RQ_TRY(qaoa_prepare(b, 1, gammas, betas));
    RQ_TRY(b->graph.run(
        b->stream, b->ev0, b->prof, [&]() { return qaoa_launch(b, 1, 0, 0, nullptr, true); },
        [&]() { return qaoa_shape(b, 1, 1, 0, 0); }));
    RQ_CUDA(cudaEventRecord(b->ev1, b->stream));
    std::vector<double> e(ninst), g((size_t)ninst * P2);
    RQ_CUDA(cudaMemcpyAsync(e.data(), b->d_energy, ninst * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    RQ_CUDA(cudaMemcpyAsync(g.data(), b->d_grad, g.size() * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    RQ_CUDA(cudaStreamSynchronize(b->stream));
    RQ_CUDA(cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
    b->graph.collect(b->prof);
    for (uint32_t k = 0; k < ninst; ++k) {
        const uint64_t user = b->order[k];
        energies[user] = e[k];
        for (uint32_t j = 0; j < P2; ++j) gradients[user * P2 + j] = g[(size_t)k * P2 + j];
    }
    b->last_nsets = 1;
    return RQ_OK;
}

}  // extern "C"

namespace {

// Adam (precond == nullptr) or preconditioned ascent (precond: ninst x 2p x 2p, caller order)
int optimize_impl(rq_qaoa_batch* b, uint32_t steps, double lr, double* gammas, double* betas, const double* target,
                  double rtol, int32_t gradient, const double* precond, double alpha0, double* energies,
                  uint32_t* steps_taken) {
    if (!b || !gammas || !betas || !energies || !steps_taken) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (precond && gradient != RQ_QAOA_GRAD_ADJOINT)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "preconditioned steps take the exact (adjoint) gradient");
    if (precond && 2 * b->p > 128) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "preconditioned steps take p <= 64");
    if (gradient != RQ_QAOA_GRAD_ADJOINT && gradient != RQ_QAOA_GRAD_SHIFT)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "gradient must be RQ_QAOA_GRAD_ADJOINT or RQ_QAOA_GRAD_SHIFT");
    RQ_CUDA(cudaSetDevice(b->device));
    const bool adj = gradient == RQ_QAOA_GRAD_ADJOINT;
    const uint32_t p = b->p, P2 = 2 * p, nsets = adj ? 1 : 1 + 2 * P2, ninst = b->ninst;
    RQ_TRY(qaoa_prepare(b, nsets, nullptr, nullptr));
    // instances in run order (class-major), angles as theta = (gammas, betas) per instance
    std::vector<uint32_t> inst_order;
    for (auto& K : b->classes)
        for (uint32_t inst : K.insts) inst_order.push_back(inst);
    std::vector<double> th((size_t)ninst * P2), tg(ninst);
    for (uint32_t r = 0; r < ninst; ++r) {
        const uint32_t i = inst_order[r];
        for (uint32_t l = 0; l < p; ++l) {
            th[(size_t)r * P2 + l] = gammas[(size_t)i * p + l];
            th[(size_t)r * P2 + p + l] = betas[(size_t)i * p + l];
        }
        if (target) tg[r] = target[i];
    }
    // run-order position of each size class's first instance
    std::vector<uint32_t> cls_of(ninst);
    {
        uint32_t r = 0;
        for (size_t k = 0; k < b->classes.size(); ++k)
            for (size_t j = 0; j < b->classes[k].insts.size(); ++j) cls_of[r++] = (uint32_t)k;
    }
    double *d_th = nullptr, *d_m = nullptr, *d_v = nullptr, *d_tg = nullptr, *d_el = nullptr;
    double *d_pre = nullptr, *d_alpha = nullptr, *d_eprev = nullptr;
    uint32_t *d_done = nullptr, *d_act = nullptr, *d_step = nullptr;
    // one optimizer step as a CUDA graph, captured per active set (after an uncaptured first
    // step has sized every buffer) and replayed until the set changes
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool use_graph = std::getenv("RUQU_NO_GRAPHS") == nullptr;
    auto drop_graph = [&]() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        gexec = nullptr;
        graph = nullptr;
    };
    auto cleanup = [&]() {
        drop_graph();
        void* q[] = {d_th, d_m, d_v, d_tg, d_el, d_done, d_act, d_step, d_pre, d_alpha, d_eprev};
        for (void* x : q) if (x) cudaFree(x);
    };
    int rc = RQ_OK;
    if (rc == RQ_OK) rc = dalloc_b(&d_th, th.size());
    if (rc == RQ_OK) rc = dalloc_b(&d_m, th.size());
    if (rc == RQ_OK) rc = dalloc_b(&d_v, th.size());
    if (rc == RQ_OK) rc = dalloc_b(&d_tg, ninst);
    if (rc == RQ_OK) rc = dalloc_b(&d_el, ninst);
    if (rc == RQ_OK) rc = dalloc_b(&d_done, ninst);
    if (rc == RQ_OK) rc = dalloc_b(&d_act, ninst);
    if (rc == RQ_OK) rc = dalloc_b(&d_step, 1);
    if (rc == RQ_OK) rc = dalloc_b(&d_eprev, ninst);
    if (precond) {
        if (rc == RQ_OK) rc = dalloc_b(&d_pre, (size_t)ninst * P2 * P2);
        if (rc == RQ_OK) rc = dalloc_b(&d_alpha, ninst);
    }
    if (rc != RQ_OK) { cleanup(); return rc; }
    std::vector<double> pre_run, alpha_init, eprev_init;
    if (precond) {   // preconditioners in run order
        pre_run.resize((size_t)ninst * P2 * P2);
        for (uint32_t r = 0; r < ninst; ++r)
            std::memcpy(&pre_run[(size_t)r * P2 * P2], precond + (size_t)inst_order[r] * P2 * P2,
                        (size_t)P2 * P2 * sizeof(double));
        alpha_init.assign(ninst, alpha0);
        cudaMemcpyAsync(d_pre, pre_run.data(), pre_run.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream);
        cudaMemcpyAsync(d_alpha, alpha_init.data(), ninst * sizeof(double), cudaMemcpyHostToDevice, b->stream);
    }
    // the previous step's energy of every instance (damping, convergence rule): none yet
    eprev_init.assign(ninst, -1e300);
    cudaMemcpyAsync(d_eprev, eprev_init.data(), ninst * sizeof(double), cudaMemcpyHostToDevice, b->stream);
    const double conv = b->conv_tol;
    // active set: run-order instances still optimising, their circuits' instance map, and per-class counts
    std::vector<uint32_t> act(ninst), ci;
    for (uint32_t r = 0; r < ninst; ++r) act[r] = r;
    std::vector<uint64_t> per_class(b->classes.size());
    std::vector<uint32_t> dn(ninst, 0);
    auto upload_active = [&]() -> int {
        std::fill(per_class.begin(), per_class.end(), 0);
        ci.clear();
        for (uint32_t r : act) {
            ++per_class[cls_of[r]];
            for (uint32_t s2 = 0; s2 < nsets; ++s2) ci.push_back(inst_order[r]);
        }
        RQ_CUDA(cudaMemcpyAsync(d_act, act.data(), act.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
        RQ_CUDA(cudaMemcpyAsync(b->d_circ_inst, ci.data(), ci.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                b->stream));
        // the pageable sources must outlive the copies
        RQ_CUDA(cudaStreamSynchronize(b->stream));
        return RQ_OK;
    };
    cudaMemcpyAsync(d_th, th.data(), th.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream);
    cudaMemsetAsync(d_m, 0, th.size() * sizeof(double), b->stream);
    cudaMemsetAsync(d_v, 0, th.size() * sizeof(double), b->stream);
    cudaMemsetAsync(d_done, 0, ninst * sizeof(uint32_t), b->stream);
    cudaMemsetAsync(d_step, 0, sizeof(uint32_t), b->stream);
    if (target) cudaMemcpyAsync(d_tg, tg.data(), ninst * sizeof(double), cudaMemcpyHostToDevice, b->stream);
    rc = upload_active();
    const int sms = rq::num_sms(b->device);
    cudaEventRecord(b->ev0, b->stream);
    // one step: shifted angles, energies (+ gradients), Adam, step counter
    auto enqueue_step = [&](bool final_eval) -> int {
        const uint32_t nact = (uint32_t)act.size();
        const uint64_t ncirc = (uint64_t)nact * nsets;
        k_qaoa_shift<<<rq::grid_for(ncirc * p, TPB, sms), TPB, 0, b->stream>>>(d_th, d_act, nact, p, nsets, b->d_ang);
        RQ_TRY(qaoa_launch(b, nsets, 0, 0, &per_class, adj && !final_eval));
        if (precond)
            k_qaoa_precond<<<rq::grid_for(nact, TPB, sms), TPB, 0, b->stream>>>(
                b->d_energy, d_act, nact, p, d_th, d_pre, d_alpha, d_eprev, target ? d_tg : nullptr, rtol, d_done,
                d_el, final_eval ? 1 : 0, b->d_grad, d_step, conv);
        else
            k_qaoa_adam<<<rq::grid_for(nact, TPB, sms), TPB, 0, b->stream>>>(b->d_energy, d_act, nact, p, nsets, d_th,
                                                                          d_m, d_v, lr, 0, target ? d_tg : nullptr,
                                                                          rtol, d_done, d_el, final_eval ? 1 : 0,
                                                                          adj ? b->d_grad : nullptr, d_step, d_eprev,
                                                                          conv);
        k_step_inc<<<1, 32, 0, b->stream>>>(d_step);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return rq::cuda_fail(e, "optimizer kernels");
        return RQ_OK;
    };
    for (uint32_t step = 0; step <= steps && rc == RQ_OK; ++step) {
        if (step == 0 || step == steps || !use_graph) {
            rc = enqueue_step(step == steps);
        } else {
            if (!gexec) {
                cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed);
                int crc = e == cudaSuccess ? enqueue_step(false) : RQ_ERR_CUDA;
                cudaGraph_t g = nullptr;
                cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
                if (crc == RQ_OK && e2 == cudaSuccess && g &&
                    cudaGraphInstantiate(&gexec, g, 0) == cudaSuccess) {
                    graph = g;
                } else {   // capture did not work here: plain launches from now on
                    if (g) cudaGraphDestroy(g);
                    gexec = nullptr;
                    use_graph = false;
                    cudaGetLastError();
                    rc = enqueue_step(false);
                    if (rc != RQ_OK) break;
                    goto polled;
                }
            }
            {
                cudaError_t e = cudaGraphLaunch(gexec, b->stream);
                if (e != cudaSuccess) { rc = rq::cuda_fail(e, "optimizer step graph"); break; }
            }
        }
    polled:
        if (rc != RQ_OK) break;
        cudaError_t e = cudaSuccess;
        if ((target || conv > 0.0) && step < steps && (step % 2 == 1)) {
            // drop the instances that met their target from the next steps' launches; the
            // rest keep their slots' math (every circuit's energy is independent of the batch)
            e = cudaMemcpyAsync(dn.data(), d_done, ninst * sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
            if (e != cudaSuccess) { rc = rq::cuda_fail(e, "optimizer poll"); break; }
            std::vector<uint32_t> still;
            for (uint32_t r : act)
                if (dn[r] == 0) still.push_back(r);
            if (still.empty()) break;
            if (still.size() < act.size()) {
                act.swap(still);
                drop_graph();   // the next step is captured again for the smaller set
                rc = upload_active();
            }
        }
    }
    cudaEventRecord(b->ev1, b->stream);
    std::vector<double> el(ninst);
    if (rc == RQ_OK) {
        cudaMemcpyAsync(th.data(), d_th, th.size() * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
        cudaMemcpyAsync(el.data(), d_el, ninst * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
        cudaMemcpyAsync(dn.data(), d_done, ninst * sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream);
        cudaError_t e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) rc = rq::cuda_fail(e, "optimizer");
        cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
    }
    cleanup();
    // the wave buffer holds shifted-angle circuits of a compacted run: nothing there for state()
    b->last_wave_count = 0;
    RQ_TRY(rc);
    for (uint32_t r = 0; r < ninst; ++r) {
        const uint32_t i = inst_order[r];
        for (uint32_t l = 0; l < p; ++l) {
            gammas[(size_t)i * p + l] = th[(size_t)r * P2 + l];
            betas[(size_t)i * p + l] = th[(size_t)r * P2 + p + l];
        }
        energies[i] = el[r];
        steps_taken[i] = dn[r] ? dn[r] - 1 : steps;
    }
    return RQ_OK;
}

}  // namespace

extern "C" {

int rq_qaoa_batch_optimize(rq_qaoa_batch* b, uint32_t steps, double lr, double* gammas, double* betas,
                           const double* target, double rtol, int32_t gradient, double* energies,
                           uint32_t* steps_taken) {
    return optimize_impl(b, steps, lr, gammas, betas, target, rtol, gradient, nullptr, 0.0, energies, steps_taken);
}

int rq_qaoa_batch_optimize_precond(rq_qaoa_batch* b, uint32_t steps, const double* precond, double alpha,
                                   double* gammas, double* betas, const double* target, double rtol,
                                   double* energies, uint32_t* steps_taken) {
    if (!precond) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (!(alpha > 0.0)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "alpha must be positive");
    return optimize_impl(b, steps, 0.0, gammas, betas, target, rtol, RQ_QAOA_GRAD_ADJOINT, precond, alpha, energies,
                         steps_taken);
}

int rq_qaoa_batch_set_convergence(rq_qaoa_batch* b, double tol) {
    if (!b) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (!(tol >= 0.0)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "tolerance must be >= 0");
    b->conv_tol = tol;
    return RQ_OK;
}

int rq_qaoa_batch_state(rq_qaoa_batch* b, uint64_t circuit, double* interleaved) {
    if (!b || !interleaved) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_CUDA(cudaSetDevice(b->device));
    uint64_t pos = UINT64_MAX;
    for (uint64_t k = 0; k < b->order.size(); ++k)
        if (b->order[k] == circuit) { pos = k; break; }
    if (pos == UINT64_MAX || pos < b->last_wave_first || pos >= b->last_wave_first + b->last_wave_count)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "circuit " + std::to_string(circuit) +
                                                     " is not held on the device (only the last wave of the last run is)");
    const uint64_t per = 1ull << b->last_wave_n;
    const size_t es = elem_size(b->prec);
    const unsigned char* src = (const unsigned char*)b->d_states + (pos - b->last_wave_first) * per * es;
    if (b->prec == RQ_F64) {
        RQ_CUDA(cudaMemcpy(interleaved, src, per * es, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp(2 * per);
        RQ_CUDA(cudaMemcpy(tmp.data(), src, per * es, cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < 2 * per; ++i) interleaved[i] = tmp[i];
    }
    return RQ_OK;
}

int rq_qaoa_batch_last_profile(const rq_qaoa_batch* b, double* out6) {
    if (!b || !out6) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    for (int k = 0; k < 3; ++k) {
        out6[2 * k] = b->prof.work[k];
        out6[2 * k + 1] = b->prof.ms[k];
    }
    return RQ_OK;
}

int rq_qaoa_batch_set_graphs(rq_qaoa_batch* b, int32_t enable) {
    if (!b) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_CUDA(cudaSetDevice(b->device));
    RQ_CUDA(cudaStreamSynchronize(b->stream));
    b->graph.drop();
    b->graph.key.clear();
    b->graph.enabled = enable != 0;
    return RQ_OK;
}

int rq_qaoa_batch_last_graph(const rq_qaoa_batch* b, int32_t* replayed, uint64_t* kernels) {
    if (!b || !replayed || !kernels) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    *replayed = b->graph.replayed ? 1 : 0;
    *kernels = b->graph.nodes;
    return RQ_OK;
}

int rq_qaoa_batch_last_ms(const rq_qaoa_batch* b, float* ms) {
    if (!b || !ms) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    *ms = b->last_ms;
    return RQ_OK;
}

int rq_qaoa_batch_set_state_budget(rq_qaoa_batch* b, uint64_t bytes) {
    if (!b || bytes == 0) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "bad argument");
    b->state_budget = bytes;
    return RQ_OK;
}

}  // extern "C"

// ===========================================================================
// batched VQE: the hardware-efficient ansatz "Ry on every qubit, then a CZ
// ladder CZ(q, q+1)" per layer, energies of a Pauli-sum Hamiltonian
// (expectation_hamiltonian, state.rs:403-408) and parameter-shift gradients
// (run_vqe's rule, vqe.rs:186-198) for many parameter sets at once.
// ===========================================================================
struct rq_vqe_batch {
    int device = 0;
    int32_t prec = RQ_F32;
    uint32_t n = 0, depth = 0, P = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<SweepDesc> descs;
    unsigned char* prog = nullptr;
    size_t off_ops = 0, smem = 0;
    uint64_t ntiles = 0;
    uint32_t m = 0;
    VGroup* d_groups = nullptr;
    VTerm* d_terms = nullptr;
    uint32_t* d_gofs = nullptr;   // groups of top pattern t: [gofs[t], gofs[t+1])
    uint32_t ngroups = 0, nterms = 0;
    uint32_t em = 0;              // log2 amplitudes of an energy tile
    double* d_part = nullptr;
    size_t part_cap = 0;
    double* d_params = nullptr;
    size_t params_cap = 0;
    void* d_rot = nullptr;
    size_t rot_cap = 0;
    void* d_states = nullptr;
    size_t states_cap = 0;
    double* d_energy = nullptr;
    size_t energy_cap = 0;
    float last_ms = 0.f;
    RunProfile prof;
    RunGraph graph;                         // rq_vqe_batch_run
    size_t wave_bytes = (size_t)96 << 20;   // states per wave kept around the L2 size
    // exact gradients: the reversed ansatz as an adjoint program, H as operator strings
    uint32_t am = 0;
    uint64_t antiles = 0;
    std::vector<SweepDesc> adescs;
    unsigned char* aprog = nullptr;
    size_t aoff_ops = 0;
    HTerm* d_hterms = nullptr;
    uint32_t nhterms = 0;
    void* d_lam = nullptr;
    size_t lam_cap = 0;
    double* d_gpart = nullptr;
    size_t gpart_cap = 0;
    double* d_grad = nullptr;
    size_t grad_cap = 0;
};

namespace {

// energy of every circuit of a wave through the tiled kernel
template <typename T>
int vqe_energy(rq_vqe_batch* b, uint64_t ncirc, uint64_t circ0) {
    using V = typename C2<T>::t;
    const uint32_t n = b->n;
    const uint32_t M = b->em;
    const uint32_t ntile = 1u << (n - M);
    const uint32_t threads = 512;
    const size_t smem = 2 * ((size_t)1 << M) * sizeof(V) + (size_t)(threads / 32) * b->nterms * sizeof(double);
    if (smem > 227 * 1024) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "Hamiltonian has too many strings for the energy kernel");
    auto kern = k_vqe_energy_tiles<T>;
    RQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    RQ_TRY(grow(&b->d_part, &b->part_cap, ncirc * ntile * std::max<uint32_t>(1, b->nterms)));
    int per_sm = 0;
    RQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)threads, smem));
    if (per_sm < 1) return rq::fail(RQ_ERR_CUDA, "energy kernel does not fit on an SM");
    const int sms = rq::num_sms(b->device);
    const unsigned grid = (unsigned)std::min<uint64_t>(ncirc * ntile, (uint64_t)sms * per_sm);
    kern<<<grid, threads, smem, b->stream>>>((const V*)b->d_states, n, M, ncirc, b->d_groups, b->d_gofs, b->nterms,
                                             b->d_terms, b->d_part);
    RQ_CUDA(cudaGetLastError());
    k_vqe_finalize<<<rq::grid_for(ncirc, TPB, sms), TPB, 0, b->stream>>>(b->d_part, ncirc, ntile, b->nterms, b->d_terms,
                                                                         circ0, b->d_energy);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

template <typename T>
int vqe_wave(rq_vqe_batch* b, uint64_t ncirc, uint64_t circ0) {
    using V = typename C2<T>::t;
    constexpr int RBc = std::is_same<T, float>::value ? 5 : 4;
    QArgs<T> a{};
    a.amps = (V*)b->d_states;
    a.ncirc = ncirc;
    a.ntiles = b->ntiles;
    a.circ0 = circ0;
    a.rot = (const T*)b->d_rot;
    a.nparam = b->P;
    const PhaseDesc* ph = reinterpret_cast<const PhaseDesc*>(b->prog);
    const SwOp* op = reinterpret_cast<const SwOp*>(b->prog + b->off_ops);
    auto kern = k_batch_sweep<T, RBc>;
    RQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem));
    const unsigned threads = 1u << (b->m - RBc);
    int per_sm = 0;
    RQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)threads, b->smem));
    if (per_sm < 1) return rq::fail(RQ_ERR_CUDA, "batched sweep kernel does not fit on an SM");
    const int sms = rq::num_sms(b->device);
    const unsigned grid = (unsigned)std::min<uint64_t>(ncirc * b->ntiles, (uint64_t)sms * per_sm);
    int ev = b->prof.begin(b->stream);
    for (const auto& d : b->descs) {
        kern<<<grid, threads, b->smem, b->stream>>>(d, ph, op, a);
        RQ_CUDA(cudaGetLastError());
    }
    const double sb = (double)((size_t)1 << b->n) * sizeof(V);
    b->prof.end(ev, b->stream, 0, (double)ncirc * sweep_bytes(b->descs, sb));
    ev = b->prof.begin(b->stream);
    RQ_TRY(vqe_energy<T>(b, ncirc, circ0));
    // per string and amplitude: one complex product conj(a[i ^ x]) a[i] (6 flops) and its
    // FP64 accumulation (2 flops)
    b->prof.end(ev, b->stream, 1, (double)ncirc * (double)b->nterms * (double)((size_t)1 << b->n) * 8.0);
    return RQ_OK;
}

// exact gradients of a wave whose final states vqe_wave left in d_states: lambda = H psi,
// then both states run backwards through the adjoint program; every Ry adds
// Im <lambda|Y_q|psi> to its parameter's entry of d_grad (zeroed by the caller)
template <typename T>
int vqe_adjoint(rq_vqe_batch* b, uint64_t ncirc, uint64_t circ0) {
    using V = typename C2<T>::t;
    constexpr int RBc = std::is_same<T, float>::value ? 4 : 3;
    const int sms = rq::num_sms(b->device);
    const uint64_t amps = ncirc << b->n;
    const unsigned hgrid = (unsigned)std::min<uint64_t>((amps + 255) / 256, (uint64_t)sms * 8);
    k_vqe_apply_h<T><<<hgrid, 256, 0, b->stream>>>((const V*)b->d_states, (V*)b->d_lam, b->n, ncirc, b->d_hterms,
                                                   b->nhterms);
    RQ_CUDA(cudaGetLastError());
    QArgs<T> a{};
    a.amps = (V*)b->d_states;
    a.lam = (V*)b->d_lam;
    a.ncirc = ncirc;
    a.ntiles = b->antiles;
    a.circ0 = circ0;
    a.rot = (const T*)b->d_rot;
    a.nparam = b->P;
    a.gpart = b->d_gpart;
    a.gwidth = b->P;
    const PhaseDesc* ph = reinterpret_cast<const PhaseDesc*>(b->aprog);
    const SwOp* op = reinterpret_cast<const SwOp*>(b->aprog + b->aoff_ops);
    auto kern = k_batch_adjoint<T, RBc>;
    const unsigned threads = 1u << (b->am - RBc);
    const unsigned ngroup = threads < 32 ? threads : threads / 32;
    const size_t smem = 2 * ((size_t)1 << b->am) * sizeof(V) + (size_t)ngroup * b->P * sizeof(double);
    if (smem > 227 * 1024) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "too many parameters for the adjoint kernel");
    RQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    RQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)threads, smem));
    if (per_sm < 1) return rq::fail(RQ_ERR_CUDA, "adjoint sweep kernel does not fit on an SM");
    const unsigned grid = (unsigned)std::min<uint64_t>(ncirc * b->antiles, (uint64_t)sms * per_sm);
    for (const auto& d : b->adescs) {
        kern<<<grid, threads, smem, b->stream>>>(d, ph, op, a);
        RQ_CUDA(cudaGetLastError());
        k_grad_finalize<<<rq::grid_for(ncirc * b->P, TPB, sms), TPB, 0, b->stream>>>(b->d_gpart, ncirc, b->antiles,
                                                                                   b->P, circ0, b->d_grad);
        RQ_CUDA(cudaGetLastError());
    }
    return RQ_OK;
}

// every kernel of one VQE run: the rotation table, then per wave the ansatz sweeps, the
// energies and (adjoint) the backward pass
int vqe_enqueue(rq_vqe_batch* b, uint64_t ncirc, uint32_t V, uint64_t wave, bool adj) {
    const uint32_t P = b->P;
    const int sms = rq::num_sms(b->device);
    if (b->prec == RQ_F32)
        k_vqe_rot<float><<<rq::grid_for(ncirc * P, TPB, sms), TPB, 0, b->stream>>>(b->d_params, ncirc, P, V, (float*)b->d_rot);
    else
        k_vqe_rot<double><<<rq::grid_for(ncirc * P, TPB, sms), TPB, 0, b->stream>>>(b->d_params, ncirc, P, V, (double*)b->d_rot);
    RQ_CUDA(cudaGetLastError());
    for (uint64_t w0 = 0; w0 < ncirc; w0 += wave) {
        const uint64_t wn = std::min<uint64_t>(wave, ncirc - w0);
        if (b->prec == RQ_F32) {
            RQ_TRY(vqe_wave<float>(b, wn, w0));
            if (adj) {
                const int ev = b->prof.begin(b->stream);
                RQ_TRY(vqe_adjoint<float>(b, wn, w0));
                b->prof.end(ev, b->stream, 2, (double)wn * (2.0 * (double)((size_t)8 << b->n) +
                                                            sweep_bytes(b->adescs, (double)((size_t)8 << b->n), 2.0)));
            }
        } else {
            RQ_TRY(vqe_wave<double>(b, wn, w0));
            if (adj) {
                const int ev = b->prof.begin(b->stream);
                RQ_TRY(vqe_adjoint<double>(b, wn, w0));
                b->prof.end(ev, b->stream, 2, (double)wn * (2.0 * (double)((size_t)16 << b->n) +
                                                            sweep_bytes(b->adescs, (double)((size_t)16 << b->n), 2.0)));
            }
        }
    }
    return RQ_OK;
}

}  // namespace

extern "C" {

int rq_vqe_batch_create(uint32_t num_qubits, uint32_t depth, const double* coeffs, const rq_pauli_op* ops,
                        const uint32_t* offsets, uint32_t nterms, int32_t precision, rq_vqe_batch** out) {
    if (!out || (!coeffs && nterms) || (!offsets && nterms)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (precision != RQ_F32 && precision != RQ_F64)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "precision must be RQ_F32 or RQ_F64");
    const uint32_t rb = precision == RQ_F32 ? 5 : 4;
    if (num_qubits < rb + 2 || num_qubits > 30)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "batched VQE takes " + std::to_string(rb + 2) + "..30 qubits");
    if (depth == 0) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "depth must be >= 1");
    std::unique_ptr<rq_vqe_batch> b(new rq_vqe_batch());
    b->prec = precision;
    b->n = num_qubits;
    b->depth = depth;
    b->P = num_qubits * depth;
    cudaGetDevice(&b->device);
    // Hamiltonian in mask form, grouped by X/Y pattern, chunks of <= 8 terms
    std::map<uint64_t, std::vector<std::pair<uint64_t, std::pair<uint32_t, double>>>> by_x;   // x -> (pmask, (ny, coeff))
    std::vector<HTerm> hterms;
    for (uint32_t k = 0; k < nterms; ++k) {
        if (offsets[k + 1] < offsets[k]) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "offsets must be non-decreasing");
        uint64_t x = 0, pm = 0;
        uint32_t ny = 0;
        for (uint32_t j = offsets[k]; j < offsets[k + 1]; ++j) {
            const uint32_t q = ops[j].qubit;
            const int o = ops[j].op;
            if (o < RQ_PAULI_I || o > RQ_PAULI_Z) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "invalid Pauli operator");
            if (o == RQ_PAULI_I) continue;
            if (q >= num_qubits) return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "Pauli factor on qubit " + std::to_string(q));
            if (o == RQ_PAULI_X || o == RQ_PAULI_Y) x ^= 1ull << q;
            if (o == RQ_PAULI_Y || o == RQ_PAULI_Z) pm ^= 1ull << q;
            if (o == RQ_PAULI_Y) ++ny;
        }
        by_x[x].push_back({pm, {ny & 3u, coeffs[k]}});
        // the adjoint pass applies the Hermitian part of H; a string whose operator
        // i^ny X^x Z^pm is anti-Hermitian (a qubit repeated within the string) has no
        // real expectation and drops out
        if (((ny + (uint32_t)__builtin_popcountll(x & pm)) & 1u) == 0) {
            const double cf = coeffs[k];
            const uint32_t r = ny & 3u;
            HTerm h{x, pm, r == 0 ? cf : (r == 2 ? -cf : 0.0), r == 1 ? cf : (r == 3 ? -cf : 0.0)};
            hterms.push_back(h);
        }
    }
    auto re_ip = [](uint32_t k) { k &= 3u; return k == 0 ? 1.0 : (k == 2 ? -1.0 : 0.0); };
    // energy tiles: two tiles (own + partner) in shared memory, 2^13 f32 / 2^12 f64 amplitudes each
    const uint32_t Mt = std::min<uint32_t>(num_qubits, precision == RQ_F32 ? 13 : 12);
    b->em = Mt;
    const uint32_t ntile = 1u << (num_qubits - Mt);
    std::vector<VGroup> groups;
    std::vector<VTerm> terms;
    std::vector<uint32_t> gofs(ntile + 1, 0);
    for (uint32_t t = 0; t < ntile; ++t) {
        gofs[t] = (uint32_t)groups.size();
        for (auto& kv : by_x) {
            const uint64_t x = kv.first;
            if ((uint32_t)(x >> Mt) != t) continue;
            const auto& list = kv.second;
            for (size_t c0 = 0; c0 < list.size(); c0 += 8) {
                VGroup G{};
                G.x = x;
                G.h = x ? 63 - __builtin_clzll(x) : 0;
                G.t0 = (uint32_t)terms.size();
                G.nt = (uint32_t)std::min<size_t>(8, list.size() - c0);
                for (uint32_t k = 0; k < G.nt; ++k) {
                    const auto& tt = list[c0 + k];
                    VTerm vt{};
                    vt.pmask = tt.first;
                    const uint32_t ny = tt.second.first;
                    const bool odd = x && (__builtin_popcountll(x & tt.first) & 1);
                    vt.odd = odd ? 1u : 0u;
                    const double f = x == 0 ? re_ip(ny) : (odd ? 2.0 * re_ip(ny + 1) : 2.0 * re_ip(ny));
                    vt.factor = tt.second.second * f;
                    terms.push_back(vt);
                }
                groups.push_back(G);
            }
        }
    }
    gofs[ntile] = (uint32_t)groups.size();
    b->ngroups = (uint32_t)groups.size();
    b->nterms = (uint32_t)terms.size();
    if (groups.empty()) groups.push_back(VGroup{});
    if (terms.empty()) terms.push_back(VTerm{});
    RQ_CUDA(cudaMalloc((void**)&b->d_gofs, gofs.size() * sizeof(uint32_t)));
    RQ_CUDA(cudaMemcpy(b->d_gofs, gofs.data(), gofs.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    RQ_CUDA(cudaMalloc((void**)&b->d_groups, groups.size() * sizeof(VGroup)));
    RQ_CUDA(cudaMemcpy(b->d_groups, groups.data(), groups.size() * sizeof(VGroup), cudaMemcpyHostToDevice));
    RQ_CUDA(cudaMalloc((void**)&b->d_terms, terms.size() * sizeof(VTerm)));
    RQ_CUDA(cudaMemcpy(b->d_terms, terms.data(), terms.size() * sizeof(VTerm), cudaMemcpyHostToDevice));
    // the ansatz program
    b->m = std::min(num_qubits, precision == RQ_F32 ? 13u : 12u);
    const uint32_t c = std::min<uint32_t>(b->m, 5);
    b->ntiles = 1ull << (num_qubits - b->m);
    b->smem = ((size_t)1 << b->m) * elem_size(precision);
    std::vector<PGate> g;
    for (uint32_t l = 0; l < depth; ++l) {
        for (uint32_t q = 0; q < num_qubits; ++q) {
            PGate r{};
            r.type = OP_RYP;
            r.q0 = q;
            r.param = (uint16_t)(l * num_qubits + q);
            g.push_back(r);
        }
        for (uint32_t q = 0; q + 1 < num_qubits; ++q) {
            PGate z{};
            z.type = OP_CZ;
            z.q0 = q;
            z.q1 = q + 1;
            g.push_back(z);
        }
    }
    auto sweeps = plan_sweeps(g, num_qubits, b->m, c);
    std::vector<PhaseDesc> phases;
    std::vector<SwOp> opsv;
    std::vector<double> mats;
    build_program(sweeps, num_qubits, b->m, c, rb, precision == RQ_F32 ? 2 : 1, b->descs, phases, opsv, mats);
    if (precision == RQ_F32) retable_f16(b->descs, phases, rb);   // the conflict-free layout (k_batch_sweep<float>)
    b->smem += max_phases(b->descs) * sizeof(PhaseDesc);   // the phase descriptors after the tile
    b->descs.front().flags |= SWEEP_INIT_ZERO;
    b->off_ops = (phases.size() * sizeof(PhaseDesc) + 255) & ~size_t(255);
    const size_t total = b->off_ops + opsv.size() * sizeof(SwOp);
    std::vector<unsigned char> host(total);
    std::memcpy(host.data(), phases.data(), phases.size() * sizeof(PhaseDesc));
    std::memcpy(host.data() + b->off_ops, opsv.data(), opsv.size() * sizeof(SwOp));
    RQ_CUDA(cudaMalloc((void**)&b->prog, total));
    RQ_CUDA(cudaMemcpy(b->prog, host.data(), total, cudaMemcpyHostToDevice));
    {
        // the adjoint program: per layer in reverse, the CZ ladder, then Ry^-1 on every qubit
        b->nhterms = (uint32_t)hterms.size();
        if (hterms.empty()) hterms.push_back(HTerm{});
        RQ_CUDA(cudaMalloc((void**)&b->d_hterms, hterms.size() * sizeof(HTerm)));
        RQ_CUDA(cudaMemcpy(b->d_hterms, hterms.data(), hterms.size() * sizeof(HTerm), cudaMemcpyHostToDevice));
        const uint32_t arb = precision == RQ_F32 ? 4 : 3;
        b->am = std::min(num_qubits, precision == RQ_F32 ? 13u : 12u);
        b->antiles = 1ull << (num_qubits - b->am);
        const uint32_t ac = std::min<uint32_t>(b->am, 5);
        std::vector<PGate> ga;
        for (uint32_t l = depth; l-- > 0;) {
            for (uint32_t q = num_qubits - 1; q-- > 0;) {
                PGate z{};
                z.type = OP_CZ;
                z.q0 = q;
                z.q1 = q + 1;
                ga.push_back(z);
            }
            for (uint32_t q = num_qubits; q-- > 0;) {
                PGate r{};
                r.type = OP_RYP;
                r.q0 = q;
                r.param = (uint16_t)(l * num_qubits + q);
                ga.push_back(r);
            }
        }
        auto asw = plan_sweeps(ga, num_qubits, b->am, ac);
        std::vector<PhaseDesc> aph;
        std::vector<SwOp> aops;
        std::vector<double> amats;
        build_program(asw, num_qubits, b->am, ac, arb, precision == RQ_F32 ? 2 : 1, b->adescs, aph, aops, amats);
        b->aoff_ops = (aph.size() * sizeof(PhaseDesc) + 255) & ~size_t(255);
        const size_t atotal = b->aoff_ops + aops.size() * sizeof(SwOp);
        std::vector<unsigned char> ah(atotal);
        std::memcpy(ah.data(), aph.data(), aph.size() * sizeof(PhaseDesc));
        std::memcpy(ah.data() + b->aoff_ops, aops.data(), aops.size() * sizeof(SwOp));
        RQ_CUDA(cudaMalloc((void**)&b->aprog, atotal));
        RQ_CUDA(cudaMemcpy(b->aprog, ah.data(), atotal, cudaMemcpyHostToDevice));
    }
    RQ_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    RQ_CUDA(cudaEventCreate(&b->ev0));
    RQ_CUDA(cudaEventCreate(&b->ev1));
    // the table copies above may return before their DMA lands (pageable sources), and the
    // batch's stream is not ordered after them: wait here, once, before any run
    RQ_CUDA(cudaDeviceSynchronize());
    *out = b.release();
    return RQ_OK;
}

int rq_vqe_batch_run(rq_vqe_batch* b, uint32_t nsets, const double* params, int32_t with_gradient, double* energies,
                     double* gradients) {
    if (!b || !params || !energies || (with_gradient && !gradients))
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (nsets == 0) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "nsets must be >= 1");
    if (with_gradient < RQ_VQE_GRAD_NONE || with_gradient > RQ_VQE_GRAD_ADJOINT)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "with_gradient must be RQ_VQE_GRAD_NONE, _SHIFT or _ADJOINT");
    RQ_CUDA(cudaSetDevice(b->device));
    const uint32_t P = b->P;
    const bool adj = with_gradient == RQ_VQE_GRAD_ADJOINT;
    const uint32_t V = with_gradient == RQ_VQE_GRAD_SHIFT ? 1 + 2 * P : 1;
    const uint64_t ncirc = (uint64_t)nsets * V;
    const size_t es = b->prec == RQ_F32 ? sizeof(float) : sizeof(double);
    RQ_TRY(grow(&b->d_params, &b->params_cap, (size_t)nsets * P));
    RQ_TRY(grow_bytes(&b->d_rot, &b->rot_cap, ncirc * P * 2 * es));
    RQ_TRY(grow(&b->d_energy, &b->energy_cap, ncirc));
    const size_t state_bytes = ((size_t)1 << b->n) * elem_size(b->prec);
    const uint64_t wave = std::max<uint64_t>(1, std::min<uint64_t>(ncirc, b->wave_bytes / state_bytes));
    RQ_TRY(grow_bytes(&b->d_states, &b->states_cap, wave * state_bytes));
    if (adj) {
        RQ_TRY(grow_bytes(&b->d_lam, &b->lam_cap, wave * state_bytes));
        RQ_TRY(grow(&b->d_gpart, &b->gpart_cap, wave * b->antiles * P));
        RQ_TRY(grow(&b->d_grad, &b->grad_cap, (size_t)nsets * P));
        RQ_CUDA(cudaMemsetAsync(b->d_grad, 0, (size_t)nsets * P * sizeof(double), b->stream));
    }
    RQ_CUDA(cudaMemcpyAsync(b->d_params, params, (size_t)nsets * P * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    RQ_TRY(b->graph.run(
        b->stream, b->ev0, b->prof, [&]() { return vqe_enqueue(b, ncirc, V, wave, adj); },
        [&]() {
            auto a = [](const void* p) { return (uint64_t)(uintptr_t)p; };
            return std::vector<uint64_t>{ncirc, V, wave, (uint64_t)adj, a(b->d_params), a(b->d_rot), a(b->d_energy),
                                         a(b->d_states), a(b->d_part), a(b->d_lam), a(b->d_gpart), a(b->d_grad)};
        }));
    RQ_CUDA(cudaEventRecord(b->ev1, b->stream));
    std::vector<double> e(ncirc);
    RQ_CUDA(cudaMemcpyAsync(e.data(), b->d_energy, ncirc * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    if (adj)
        RQ_CUDA(cudaMemcpyAsync(gradients, b->d_grad, (size_t)nsets * P * sizeof(double), cudaMemcpyDeviceToHost,
                                b->stream));
    RQ_CUDA(cudaStreamSynchronize(b->stream));
    RQ_CUDA(cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
    b->graph.collect(b->prof);
    for (uint32_t s = 0; s < nsets; ++s) {
        energies[s] = e[(uint64_t)s * V];
        if (with_gradient == RQ_VQE_GRAD_SHIFT)
            for (uint32_t k = 0; k < P; ++k)
                gradients[(uint64_t)s * P + k] = (e[(uint64_t)s * V + 1 + 2 * k] - e[(uint64_t)s * V + 2 + 2 * k]) / 2.0;
    }
    return RQ_OK;
}


int rq_vqe_batch_last_profile(const rq_vqe_batch* b, double* out6) {
    if (!b || !out6) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    for (int k = 0; k < 3; ++k) {
        out6[2 * k] = b->prof.work[k];
        out6[2 * k + 1] = b->prof.ms[k];
    }
    return RQ_OK;
}

int rq_vqe_batch_set_graphs(rq_vqe_batch* b, int32_t enable) {
    if (!b) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_CUDA(cudaSetDevice(b->device));
    RQ_CUDA(cudaStreamSynchronize(b->stream));
    b->graph.drop();
    b->graph.key.clear();
    b->graph.enabled = enable != 0;
    return RQ_OK;
}

int rq_vqe_batch_last_graph(const rq_vqe_batch* b, int32_t* replayed, uint64_t* kernels) {
    if (!b || !replayed || !kernels) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    *replayed = b->graph.replayed ? 1 : 0;
    *kernels = b->graph.nodes;
    return RQ_OK;
}

int rq_vqe_batch_last_ms(const rq_vqe_batch* b, float* ms) {
    if (!b || !ms) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    *ms = b->last_ms;
    return RQ_OK;
}

int rq_vqe_batch_destroy(rq_vqe_batch* b) {
    if (!b) return RQ_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    void* ptrs[] = {b->prog,     b->d_groups, b->d_terms, b->d_gofs,  b->d_part, b->d_params, b->d_rot,
                    b->d_states, b->d_energy, b->aprog,   b->d_hterms, b->d_lam,  b->d_gpart,  b->d_grad};
    for (void* q : ptrs) if (q) cudaFree(q);
    b->graph.drop();
    b->prof.release();
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return RQ_OK;
}

}  // extern "C"
