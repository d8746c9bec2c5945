// rq_sweep.cu -- multi-gate sweeps: many gates per HBM pass.
//
// The reference applies every gate as its own full pass over the state
// (state.rs:214-276, called once per gate from simulator.rs:69-79).  Here a
// host planner cuts the gate list into sweeps.  A sweep owns a set L of m
// "local" qubits (always including qubits 0..c-1, so every HBM access is a
// contiguous 2^c-amplitude chunk); each CTA loads one 2^m-amplitude tile
// (all combinations of the local bits for one value of the other bits) into
// shared memory with coalesced 16-byte loads, runs the sweep's gates on it,
// and writes it back: 2*S bytes of HBM traffic per sweep instead of per gate.
//
// Inside a tile the gates run in phases.  In a phase every thread holds 2^RB
// amplitudes in registers whose indices differ in RB chosen local bits (the
// phase's register slots); a non-diagonal 1-qubit gate or a CNOT target must
// sit on a register slot, diagonal gates (Rz, Phase, S, T, Z, CZ, Rzz) and
// CNOT controls may sit on any bit because they only read index bits.
// Between phases the tile goes back through shared memory (XOR-swizzled so
// the strided reads of any slot choice stay nearly bank-conflict free).
// Adjacent 1-qubit gates on the same qubit are multiplied into one 2x2 on
// the host (a generalisation of optimizer::fuse_gates, optimizer.rs:46-94).
#include "rq_internal.cuh"
#include "rq_plan.cuh"

#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

namespace {

using rqd::C2;
using namespace rqp;

// 16-byte vector type per precision: 2 complex f32 or 1 complex f64
template <typename T> struct Vec16;
template <> struct Vec16<float> { using t = float4; static constexpr int EPV = 2; };
template <> struct Vec16<double> { using t = double2; static constexpr int EPV = 1; };

template <typename T>
__device__ __forceinline__ uint32_t swz(uint32_t e) {
    // 128-byte rows: 16 complex f32 or 8 complex f64 per row
    constexpr int CB = sizeof(typename C2<T>::t) == 8 ? 4 : 3;
    uint32_t r = e >> CB;
    uint32_t f = r ^ (r >> CB) ^ (r >> (2 * CB)) ^ (r >> (3 * CB));
    return e ^ (f & ((1u << CB) - 1));
}

template <typename V, typename T>
__device__ __forceinline__ V cmul(V a, T br, T bi) {
    V r;
    r.x = a.x * br - a.y * bi;
    r.y = a.x * bi + a.y * br;
    return r;
}

template <int K, int NR, typename V, typename T>
__device__ __forceinline__ void op_u1(V* reg, const T* __restrict__ m) {
    const T m00r = m[0], m00i = m[1], m01r = m[2], m01i = m[3];
    const T m10r = m[4], m10i = m[5], m11r = m[6], m11i = m[7];
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (i & (1 << K)) continue;
        const int j = i | (1 << K);
        V x = reg[i], y = reg[j];
        V o0, o1;
        o0.x = m00r * x.x - m00i * x.y + m01r * y.x - m01i * y.y;
        o0.y = m00r * x.y + m00i * x.x + m01r * y.y + m01i * y.x;
        o1.x = m10r * x.x - m10i * x.y + m11r * y.x - m11i * y.y;
        o1.y = m10r * x.y + m10i * x.x + m11r * y.y + m11i * y.x;
        reg[i] = o0;
        reg[j] = o1;
    }
}

// CNOT with its target on slot K; control = slot ck (>=0) or uniform bit cu
template <int K, int NR, typename V>
__device__ __forceinline__ void op_cx(V* reg, int ck, int cu) {
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (i & (1 << K)) continue;
        const int j = i | (1 << K);
        const bool c = ck >= 0 ? ((i >> ck) & 1) : cu;
        V x = reg[i], y = reg[j];
        reg[i] = c ? y : x;
        reg[j] = c ? x : y;
    }
}

template <int NR, typename V, typename T>
__device__ __forceinline__ void dispatch_u1(int k, V* reg, const T* m) {
    switch (k) {
        case 0: op_u1<0, NR>(reg, m); break;
        case 1: op_u1<1, NR>(reg, m); break;
        case 2: op_u1<2, NR>(reg, m); break;
        case 3: if constexpr (NR > 8) op_u1<3, NR>(reg, m); break;
        case 4: if constexpr (NR > 16) op_u1<4, NR>(reg, m); break;
        default: break;
    }
}

template <int NR, typename V>
__device__ __forceinline__ void dispatch_cx(int k, V* reg, int ck, int cu) {
    switch (k) {
        case 0: op_cx<0, NR>(reg, ck, cu); break;
        case 1: op_cx<1, NR>(reg, ck, cu); break;
        case 2: op_cx<2, NR>(reg, ck, cu); break;
        case 3: if constexpr (NR > 8) op_cx<3, NR>(reg, ck, cu); break;
        case 4: if constexpr (NR > 16) op_cx<4, NR>(reg, ck, cu); break;
        default: break;
    }
}

// The phases of one sweep on a tile held in shared memory (all threads of the CTA).
template <typename T, int RB>
__device__ __forceinline__ void run_phases(typename C2<T>::t* sm, const SweepDesc& d,
                                           const PhaseDesc* __restrict__ phases, const SwOp* __restrict__ ops,
                                           const T* __restrict__ mats, uint64_t base, uint32_t tid) {
    using V = typename C2<T>::t;
    constexpr int NR = 1 << RB;
    for (uint32_t p = d.phase_begin; p < d.phase_end; ++p) {
        const PhaseDesc& ph = phases[p];
        uint32_t ebase = 0;
        uint64_t U = base;
        for (uint32_t b = 0; b < ph.nt; ++b)
            if ((tid >> b) & 1u) {
                ebase |= 1u << ph.tbit_local[b];
                U |= 1ull << ph.tbit_global[b];
            }
        const uint32_t sb = swz<T>(ebase);
        V reg[NR];
#pragma unroll
        for (int i = 0; i < NR; ++i) reg[i] = sm[sb ^ ph.slut[i]];

        for (uint32_t o = ph.op_begin; o < ph.op_end; ++o) {
            const SwOp op = ops[o];
            const T* mm = mats + 2 * op.mat;
            switch (op.type) {
                case OP_U1: dispatch_u1<NR>(op.k0, reg, mm); break;
                case OP_CX: dispatch_cx<NR>(op.k1, reg, op.k0, (int)((U >> op.q0) & 1ull)); break;
                case OP_D1: {
                    const T d0r = mm[0], d0i = mm[1], d1r = mm[2], d1i = mm[3];
                    const int kk = op.k0;
                    const int ub = (int)((U >> op.q0) & 1ull);
#pragma unroll
                    for (int i = 0; i < NR; ++i) {
                        const int b = kk >= 0 ? ((i >> kk) & 1) : ub;
                        reg[i] = cmul(reg[i], b ? d1r : d0r, b ? d1i : d0i);
                    }
                    break;
                }
                case OP_CZ: {
                    const int k0 = op.k0, k1 = op.k1;
                    const int u0 = (int)((U >> op.q0) & 1ull), u1 = (int)((U >> op.q1) & 1ull);
#pragma unroll
                    for (int i = 0; i < NR; ++i) {
                        const int b0 = k0 >= 0 ? ((i >> k0) & 1) : u0;
                        const int b1 = k1 >= 0 ? ((i >> k1) & 1) : u1;
                        if (b0 & b1) {
                            reg[i].x = -reg[i].x;
                            reg[i].y = -reg[i].y;
                        }
                    }
                    break;
                }
                case OP_ZZ: {
                    // diag(en, ep, ep, en): en for equal bits, ep for different bits
                    const T er = mm[0], ei = mm[1], pr = mm[2], pi = mm[3];
                    const int k0 = op.k0, k1 = op.k1;
                    const int u0 = (int)((U >> op.q0) & 1ull), u1 = (int)((U >> op.q1) & 1ull);
#pragma unroll
                    for (int i = 0; i < NR; ++i) {
                        const int b0 = k0 >= 0 ? ((i >> k0) & 1) : u0;
                        const int b1 = k1 >= 0 ? ((i >> k1) & 1) : u1;
                        const bool diff = (b0 ^ b1) != 0;
                        reg[i] = cmul(reg[i], diff ? pr : er, diff ? pi : ei);
                    }
                    break;
                }
                default: break;
            }
        }
#pragma unroll
        for (int i = 0; i < NR; ++i) sm[sb ^ ph.slut[i]] = reg[i];
        __syncthreads();
    }
}

// Variant of run_phases: register addresses composed by XOR from the five slot
// offsets (no table loads), and the next op and its matrix fetched while the
// current op runs.
template <typename T, int RB>
__device__ __forceinline__ void run_phases_v1(typename C2<T>::t* sm, const SweepDesc& d,
                                           const PhaseDesc* __restrict__ phases, const SwOp* __restrict__ ops,
                                           const T* __restrict__ mats, uint64_t base, uint32_t tid) {
    using V = typename C2<T>::t;
    constexpr int NR = 1 << RB;
    for (uint32_t p = d.phase_begin; p < d.phase_end; ++p) {
        const PhaseDesc& ph = phases[p];
        uint32_t ebase = 0;
        uint64_t U = base;
        for (uint32_t b = 0; b < ph.nt; ++b)
            if ((tid >> b) & 1u) {
                ebase |= 1u << ph.tbit_local[b];
                U |= 1ull << ph.tbit_global[b];
            }
        const uint32_t sb = swz<T>(ebase);
        uint32_t S[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k) S[k] = ph.slut[1 << k];
        auto addr = [&](int i) {
            uint32_t a = sb;
#pragma unroll
            for (int k = 0; k < RB; ++k)
                if ((i >> k) & 1) a ^= S[k];
            return a;
        };
        V reg[NR];
#pragma unroll
        for (int i = 0; i < NR; ++i) reg[i] = sm[addr(i)];

        SwOp nop = ops[ph.op_begin];
        T nm[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) nm[k] = mats[2 * nop.mat + k];
        for (uint32_t o = ph.op_begin; o < ph.op_end; ++o) {
            const SwOp op = nop;
            T mm[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) mm[k] = nm[k];
            if (o + 1 < ph.op_end) {
                nop = ops[o + 1];
#pragma unroll
                for (int k = 0; k < 8; ++k) nm[k] = mats[2 * nop.mat + k];
            }
            switch (op.type) {
                case OP_U1: dispatch_u1<NR>(op.k0, reg, mm); break;
                case OP_CX: dispatch_cx<NR>(op.k1, reg, op.k0, (int)((U >> op.q0) & 1ull)); break;
                case OP_D1: {
                    const T d0r = mm[0], d0i = mm[1], d1r = mm[2], d1i = mm[3];
                    const int kk = op.k0;
                    const int ub = (int)((U >> op.q0) & 1ull);
#pragma unroll
                    for (int i = 0; i < NR; ++i) {
                        const int b = kk >= 0 ? ((i >> kk) & 1) : ub;
                        reg[i] = cmul(reg[i], b ? d1r : d0r, b ? d1i : d0i);
                    }
                    break;
                }
                case OP_CZ: {
                    const int k0 = op.k0, k1 = op.k1;
                    const int u0 = (int)((U >> op.q0) & 1ull), u1 = (int)((U >> op.q1) & 1ull);
#pragma unroll
                    for (int i = 0; i < NR; ++i) {
                        const int b0 = k0 >= 0 ? ((i >> k0) & 1) : u0;
                        const int b1 = k1 >= 0 ? ((i >> k1) & 1) : u1;
                        if (b0 & b1) {
                            reg[i].x = -reg[i].x;
                            reg[i].y = -reg[i].y;
                        }
                    }
                    break;
                }
                case OP_ZZ: {
                    // diag(en, ep, ep, en): en for equal bits, ep for different bits
                    const T er = mm[0], ei = mm[1], pr = mm[2], pi = mm[3];
                    const int k0 = op.k0, k1 = op.k1;
                    const int u0 = (int)((U >> op.q0) & 1ull), u1 = (int)((U >> op.q1) & 1ull);
#pragma unroll
                    for (int i = 0; i < NR; ++i) {
                        const int b0 = k0 >= 0 ? ((i >> k0) & 1) : u0;
                        const int b1 = k1 >= 0 ? ((i >> k1) & 1) : u1;
                        const bool diff = (b0 ^ b1) != 0;
                        reg[i] = cmul(reg[i], diff ? pr : er, diff ? pi : ei);
                    }
                    break;
                }
                default: break;
            }
        }
#pragma unroll
        for (int i = 0; i < NR; ++i) sm[addr(i)] = reg[i];
        __syncthreads();
    }
}

template <typename T, int RB, bool PV>
__global__ void __launch_bounds__(256, 2) k_sweep(typename C2<T>::t* __restrict__ amps, const SweepDesc d,
                                               const PhaseDesc* __restrict__ phases, const SwOp* __restrict__ ops,
                                               const T* __restrict__ mats, uint64_t ntiles) {
    using V = typename C2<T>::t;
    using VV = typename Vec16<T>::t;
    constexpr int NR = 1 << RB;
    constexpr int EPV = Vec16<T>::EPV;
    constexpr int VPT = NR / EPV;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* sm = reinterpret_cast<V*>(smem_raw);

    const uint32_t tid = threadIdx.x;
    const uint64_t cmask = (1ull << d.c) - 1;

    // deposit of this thread's vector offset (local bits of EPV*tid) into global positions
    uint64_t dep_tid = 0;
    {
        uint64_t x = (uint64_t)tid * EPV;
        dep_tid = x & cmask;
        for (uint32_t b = d.c; b < d.m; ++b)
            if ((x >> b) & 1ull) dep_tid |= 1ull << d.local_global[b];
    }
    const uint32_t stid = swz<T>(tid * EPV);   // swz(e) = stid ^ sgj[j] (the swizzle is XOR-linear)

    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        uint64_t base = 0;
        for (uint32_t b = 0; b < d.nonlocal_count; ++b)
            if ((tile >> b) & 1ull) base |= 1ull << d.nonlocal[b];

        // ---- load tile (coalesced 16-byte vectors, 8 in flight per thread) ----
#pragma unroll 1
        for (int j0 = 0; j0 < VPT; j0 += 8) {
            VV v[8];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj)
                v[jj] = __ldcs(reinterpret_cast<const VV*>(amps + (base | dep_tid | d.gj[j0 + jj])));
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
                const uint32_t se = stid ^ d.sgj[j0 + jj];
                if constexpr (EPV == 2) {
                    sm[se] = make_float2(v[jj].x, v[jj].y);
                    sm[se ^ 1u] = make_float2(v[jj].z, v[jj].w);
                } else {
                    sm[se] = *reinterpret_cast<V*>(&v[jj]);
                }
            }
        }
        __syncthreads();

        // ---- phases ----
        if (PV) run_phases_v1<T, RB>(sm, d, phases, ops, mats, base, tid);
        else run_phases<T, RB>(sm, d, phases, ops, mats, base, tid);

        // ---- store tile ----
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            const uint32_t se = stid ^ d.sgj[j];
            const uint64_t g = base | dep_tid | d.gj[j];
            VV v;
            if constexpr (EPV == 2) {
                float2 a = sm[se], b = sm[se ^ 1u];
                v = make_float4(a.x, a.y, b.x, b.y);
            } else {
                V a = sm[se];
                v = *reinterpret_cast<VV*>(&a);
            }
            __stcs(reinterpret_cast<VV*>(amps + g), v);
        }
        __syncthreads();
    }
}

// Asynchronous global -> shared copies (cp.async): the data bypasses registers,
// so the next tile streams in while the CTA computes on the current one.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Tile loads of one thread into a swizzled shared-memory buffer: the element
// granularity of the swizzle is kept (f32: two 8-byte copies per 16-byte vector).
template <typename T>
__device__ __forceinline__ void issue_tile(typename C2<T>::t* buf, const typename C2<T>::t* __restrict__ amps,
                                           const SweepDesc& d, uint64_t base, uint64_t dep_tid, uint32_t stid) {
    constexpr int EPV = Vec16<T>::EPV;
    constexpr int VPT = (1 << (std::is_same<T, float>::value ? 5 : 4)) / EPV;
#pragma unroll
    for (int j = 0; j < VPT; ++j) {
        const typename C2<T>::t* g = amps + (base | dep_tid | d.gj[j]);
        const uint32_t se = stid ^ d.sgj[j];
        if constexpr (EPV == 2) {
            cp_async8(buf + se, g);
            cp_async8(buf + (se ^ 1u), g + 1);
        } else {
            cp_async16(buf + se, g);
        }
    }
}

// Persistent, double-buffered sweep: one CTA per SM walks tiles blockIdx.x,
// blockIdx.x + gridDim.x, ...; the copies of tile k+1 are in flight while the
// phases of tile k run and its stores drain.
template <typename T, int RB, bool PV>
__global__ void __launch_bounds__(256, 1) k_sweep_pipe(typename C2<T>::t* __restrict__ amps, const SweepDesc d,
                                                     const PhaseDesc* __restrict__ phases,
                                                     const SwOp* __restrict__ ops, const T* __restrict__ mats,
                                                     uint64_t ntiles) {
    using V = typename C2<T>::t;
    using VV = typename Vec16<T>::t;
    constexpr int NR = 1 << RB;
    constexpr int EPV = Vec16<T>::EPV;
    constexpr int VPT = NR / EPV;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* buf0 = reinterpret_cast<V*>(smem_raw);
    V* buf1 = buf0 + (1u << d.m);

    const uint32_t tid = threadIdx.x;
    const uint64_t cmask = (1ull << d.c) - 1;
    uint64_t dep_tid = 0;
    {
        uint64_t x = (uint64_t)tid * EPV;
        dep_tid = x & cmask;
        for (uint32_t b = d.c; b < d.m; ++b)
            if ((x >> b) & 1ull) dep_tid |= 1ull << d.local_global[b];
    }
    const uint32_t stid = swz<T>(tid * EPV);
    auto tile_base = [&](uint64_t tile) {
        uint64_t base = 0;
        for (uint32_t b = 0; b < d.nonlocal_count; ++b)
            if ((tile >> b) & 1ull) base |= 1ull << d.nonlocal[b];
        return base;
    };

    uint64_t tile = blockIdx.x;
    if (tile < ntiles) issue_tile<T>(buf0, amps, d, tile_base(tile), dep_tid, stid);
    cp_async_commit();
    bool cur1 = false;
    for (; tile < ntiles; tile += gridDim.x) {
        V* sm = cur1 ? buf1 : buf0;
        V* nx = cur1 ? buf0 : buf1;
        const uint64_t next = tile + gridDim.x;
        if (next < ntiles) issue_tile<T>(nx, amps, d, tile_base(next), dep_tid, stid);
        cp_async_commit();
        cp_async_wait1();          // this thread's copies of the current tile have landed
        __syncthreads();           // ... and everyone else's
        const uint64_t base = tile_base(tile);
        if (PV) run_phases_v1<T, RB>(sm, d, phases, ops, mats, base, tid);
        else run_phases<T, RB>(sm, d, phases, ops, mats, base, tid);
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            const uint32_t se = stid ^ d.sgj[j];
            const uint64_t g = base | dep_tid | d.gj[j];
            VV v;
            if constexpr (EPV == 2) {
                float2 a = sm[se], b = sm[se ^ 1u];
                v = make_float4(a.x, a.y, b.x, b.y);
            } else {
                V a = sm[se];
                v = *reinterpret_cast<VV*>(&a);
            }
            __stcs(reinterpret_cast<VV*>(amps + g), v);
        }
        __syncthreads();           // the buffer is free for the copies issued next iteration
        cur1 = !cur1;
    }
    cp_async_wait0();
}

// ---------------------------------------------------------------------------
// Tensor-core sweeps: dense 32x32 phase unitaries as TF32 MMAs (tcgen05)
// ---------------------------------------------------------------------------
//
// Complex f32 states, m = 13 local qubits (256 threads x 32 register
// amplitudes) or m = 12 (128 threads); two CTAs per SM, so one CTA's copies
// and MMAs overlap the other's CUDA-core work.  The sweep's phase and op
// descriptors are copied into shared memory at the start.  At the start of a
// phase whose first op is an OP_DENSE, one thread starts a bulk copy of the
// op's operand image (B, 64x64 TF32 values, plus the FP32 remainder for 3
// passes) into shared memory.  The dense op: every thread stores its 32
// amplitudes (64 floats: re, im of register amplitude 0, 1, ...) into its own
// tensor-memory lane as row n = tid of the A operand (TF32 high part); one
// thread issues, per 128-row half, the K = 64 products in steps of 8 into a
// 128 x 64 FP32 accumulator; for 3xTF32 the same A is multiplied by the
// image's remainder, then A is overwritten with the FP32 remainder of the
// amplitudes and multiplied by the high image; tcgen05.commit signals an
// mbarrier and every thread reads its row of the accumulator back
// (tcgen05.ld) as its 32 new amplitudes.  Tensor memory (256 columns per CTA):
// accumulator [0, 128), A [128, 256); half h of the rows uses columns 64h..
namespace tc {

constexpr uint32_t B_SBO = 2048;   // bytes between 8-row groups of an image (16 core matrices along K)
constexpr uint32_t B_LBO = 128;    // bytes between core matrices along K
constexpr uint32_t COL_D = 0;   // accumulator columns [0, 64 * halves); A follows at col_a = 64 * halves

__device__ int g_tc_timeout = 0;
// polls of an mbarrier before a main-path wait counts as expired (rq_debug_set_wait_limit);
// the clean-up waits after an expiry always use WAIT_POLLS
constexpr uint32_t WAIT_POLLS = 1u << 24;
__device__ uint32_t g_tc_wait_polls = WAIT_POLLS;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)(B_LBO >> 4) << 16;
    d |= (uint64_t)(B_SBO >> 4) << 32;
    d |= (uint64_t)1 << 46;   // sm_100 descriptor version; no swizzle, base offset 0
    return d;
}

// TF32 x TF32 -> F32, both operands K-major, M = 128, N = 64
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t polls = WAIT_POLLS) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < polls; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// round to the nearest TF32 value (ties away from zero) with integer operations: add half
// a unit of the 10-bit mantissa to the magnitude bits and clear the 13 low bits (amplitudes
// are finite; the carry into the exponent is the correct rounding)
__device__ __forceinline__ float to_tf32(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// 16 accumulator columns of this thread's lane -> 8 complex amplitudes
__device__ __forceinline__ void ld16(uint32_t taddr, float2* out) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int j = 0; j < 8; ++j) out[j] = make_float2(__uint_as_float(r[2 * j]), __uint_as_float(r[2 * j + 1]));
}

__device__ __forceinline__ void st16(uint32_t taddr, const float* v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
        ::"r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
        "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
        "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
        "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
        "r"(__float_as_uint(v[15]))
        : "memory");
}

struct TcCtx {
    float* img;          // shared-memory image buffer
    uint32_t img_bytes;  // bytes copied per image (1 pass: high part only)
    uint64_t* bar;       // MMA completion
    uint64_t* ibar;      // image copy completion
    uint32_t tmem;
    uint32_t col_a;      // first column of A (64 per 128-row half after the accumulator)
    uint32_t parity, iparity;
    int passes;
    bool failed;
};

// thread 0: bulk copy of one operand image into shared memory, completion on ibar
__device__ __forceinline__ void start_image(TcCtx& c, const float* src) {
    const uint32_t b = smem_u32(c.ibar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(c.img_bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(c.img)),
                 "l"(src), "r"(c.img_bytes), "r"(b)
                 : "memory");
}

__device__ __forceinline__ void store_a(TcCtx& c, const float2* reg, uint32_t taddr, bool low) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float h[16];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float2 v = reg[8 * q + j];
            const float hx = to_tf32(v.x), hy = to_tf32(v.y);
            h[2 * j] = low ? v.x - hx : hx;
            h[2 * j + 1] = low ? v.y - hy : hy;
        }
        st16(taddr + 16 * q, h);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// thread 0: the products of A (tensor memory) with one image part, into the accumulator
__device__ __forceinline__ void issue(TcCtx& c, uint32_t bsmem, uint32_t halves, bool first) {
    for (uint32_t h = 0; h < halves; ++h)
        for (int ks = 0; ks < 8; ++ks) {
            const uint64_t bd = sdesc(bsmem + ks * 2 * B_LBO);
            const uint32_t acc = (!first || ks > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                ::"r"(c.tmem + COL_D + h * 64), "r"(c.tmem + c.col_a + h * 64 + ks * 8), "l"(bd), "r"(IDESC),
                "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                : "memory");
        }
}

// waits on the MMA barrier; a wait that runs out marks the CTA failed (uniformly)
__device__ __forceinline__ bool commit_wait(TcCtx& c, uint32_t tid) {
    if (tid == 0)
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(c.bar))
                     : "memory");
    const bool late = !mbar_wait(c.bar, c.parity, g_tc_wait_polls);
    c.parity ^= 1u;
    if (__syncthreads_or(late)) {
        c.failed = true;
        if (tid == 0) g_tc_timeout = 1;
        return false;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return true;
}

// One OP_DENSE on the CTA's registers.  All threads call it (uniform control flow).
__device__ __forceinline__ void dense_op(TcCtx& c, float2* reg, uint32_t tid, uint32_t nthreads) {
    const uint32_t warp = tid >> 5;
    const uint32_t lane_base = ((warp & 3u) * 32u) << 16;
    const uint32_t half_col = (warp >> 2) * 64u;
    const uint32_t halves = nthreads / 128;
    store_a(c, reg, c.tmem + lane_base + c.col_a + half_col, false);
    // the image copy started at the phase start
    const bool late = !mbar_wait(c.ibar, c.iparity, g_tc_wait_polls);
    c.iparity ^= 1u;
    if (__syncthreads_or(late)) {
        c.failed = true;
        if (tid == 0) g_tc_timeout = 1;
        return;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t bhi = smem_u32(c.img), blo = smem_u32(c.img + DENSE_FLOATS);
    if (tid == 0) {
        issue(c, bhi, halves, true);
        if (c.passes > 1) issue(c, blo, halves, false);
    }
    if (!commit_wait(c, tid)) return;
    if (c.passes > 1) {
        store_a(c, reg, c.tmem + lane_base + c.col_a + half_col, true);
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) issue(c, bhi, halves, false);
        if (!commit_wait(c, tid)) return;
    }
    const uint32_t taddr = c.tmem + lane_base + COL_D + half_col;
    ld16(taddr, reg);
    ld16(taddr + 16, reg + 8);
    ld16(taddr + 32, reg + 16);
    ld16(taddr + 48, reg + 24);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

}  // namespace tc

// run_phases for the tensor-core sweep (complex f32, RB = 5).  With every gate
// qubit planned onto a register slot, each phase of such a plan is exactly
// one OP_DENSE (the planner checks this).
__device__ __forceinline__ void run_phases_tc(float2* sm, const SweepDesc& d, const PhaseDesc* phases,
                                              const SwOp* ops, const float* __restrict__ images, uint64_t base,
                                              uint32_t tid, uint32_t nthreads, tc::TcCtx& c) {
    using V = float2;
    constexpr int NR = 32;
    for (uint32_t p = d.phase_begin; p < d.phase_end; ++p) {
        const PhaseDesc& ph = phases[p];
        if (tid == 0) {
            // the image variant for this tile's values of the phase's qubits outside the tile
            const SwOp& op = ops[ph.op_begin];
            uint32_t var = 0;
            for (int j = 0; j < dense_nvq(op); ++j) var |= (uint32_t)((base >> dense_vq(op, j)) & 1ull) << j;
            tc::start_image(c, images + (size_t)(op.mat + var) * DENSE_IMAGE_FLOATS);
        }
        uint32_t ebase = 0;
        for (uint32_t b = 0; b < ph.nt; ++b)
            if ((tid >> b) & 1u) ebase |= 1u << ph.tbit_local[b];
        const uint32_t sb = swz<float>(ebase);
        // register addresses: XOR combinations of the five slot offsets (read again for the store,
        // after the dense op, so that they are not held across it)
        auto addr = [&](int i, const uint32_t* S) {
            uint32_t a = sb;
#pragma unroll
            for (int k = 0; k < 5; ++k)
                if ((i >> k) & 1) a ^= S[k];
            return a;
        };
        V reg[NR];
        {
            uint32_t S[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) S[k] = ph.slut[1 << k];
#pragma unroll
            for (int i = 0; i < NR; ++i) reg[i] = sm[addr(i, S)];
        }
        tc::dense_op(c, reg, tid, nthreads);
        if (c.failed) return;
        {
            uint32_t S[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) S[k] = ph.slut[1 << k];
#pragma unroll
            for (int i = 0; i < NR; ++i) sm[addr(i, S)] = reg[i];
        }
        __syncthreads();
    }
}

// Tensor-core sweep kernel, persistent over tiles, two CTAs per SM.  Shared
// memory: tile | image buffer | the sweep's phase and op descriptors.  Tensor
// memory is allocated once per CTA and always freed, also after a timed-out wait.
__global__ void __launch_bounds__(256, 2) k_sweep_tc(float2* __restrict__ amps, const SweepDesc d,
                                                   const PhaseDesc* __restrict__ phases, const SwOp* __restrict__ ops,
                                                   const float* __restrict__ mats, const float* __restrict__ images,
                                                   uint64_t ntiles, int passes) {
    using V = float2;
    using VV = float4;
    constexpr int EPV = 2;
    constexpr int VPT = 32 / EPV;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t tile_elems = 1u << d.m;
    V* sm = reinterpret_cast<V*>(smem_raw);
    float* img = reinterpret_cast<float*>(sm + tile_elems);
    const uint32_t img_bytes = (passes > 1 ? DENSE_IMAGE_FLOATS : DENSE_FLOATS) * 4u;
    PhaseDesc* sph = reinterpret_cast<PhaseDesc*>(reinterpret_cast<unsigned char*>(img) + img_bytes);
    const uint32_t nph = d.phase_end - d.phase_begin;
    const uint32_t op0 = phases[d.phase_begin].op_begin, nops = phases[d.phase_end - 1].op_end - op0;
    SwOp* sop = reinterpret_cast<SwOp*>(sph + nph);
    __shared__ __align__(8) uint64_t bar, ibar;
    __shared__ uint32_t tmem_base;

    const uint32_t tid = threadIdx.x;
    const uint32_t T_ = blockDim.x;
    for (uint32_t k = tid; k < nph * (uint32_t)(sizeof(PhaseDesc) / 16); k += T_)
        reinterpret_cast<uint4*>(sph)[k] = reinterpret_cast<const uint4*>(phases + d.phase_begin)[k];
    for (uint32_t k = tid; k < nops; k += T_) sop[k] = ops[op0 + k];
    tc::TcCtx c;
    c.img = img;
    c.img_bytes = img_bytes;
    c.bar = &bar;
    c.ibar = &ibar;
    c.parity = 0;
    c.iparity = 0;
    c.passes = passes;
    c.failed = false;
    // tensor memory: accumulator and A, 64 columns each per 128-row half
    const uint32_t ncols = 128u * (T_ / 128u);
    c.col_a = 64u * (T_ / 128u);
    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(&tmem_base)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc::smem_u32(&bar)), "r"(1u) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc::smem_u32(&ibar)), "r"(1u) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    c.tmem = tmem_base;
    const PhaseDesc* lph = sph - d.phase_begin;   // indexable by the sweep's global phase numbers
    const SwOp* lop = sop - op0;

    const uint64_t cmask = (1ull << d.c) - 1;
    uint64_t dep_tid = 0;
    {
        uint64_t x = (uint64_t)tid * EPV;
        dep_tid = x & cmask;
        for (uint32_t b = d.c; b < d.m; ++b)
            if ((x >> b) & 1ull) dep_tid |= 1ull << d.local_global[b];
    }
    const uint32_t stid = swz<float>(tid * EPV);

    for (uint64_t tile = blockIdx.x; tile < ntiles && !c.failed; tile += gridDim.x) {
        uint64_t base = 0;
        for (uint32_t b = 0; b < d.nonlocal_count; ++b)
            if ((tile >> b) & 1ull) base |= 1ull << d.nonlocal[b];
        // all of the tile's copies in flight at once (cp.async, element-granular for the swizzle)
        issue_tile<float>(sm, amps, d, base, dep_tid, stid);
        cp_async_commit();
        cp_async_wait0();
        __syncthreads();
        run_phases_tc(sm, d, lph, lop, images, base, tid, T_, c);
        if (c.failed) break;
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            const uint32_t se = stid ^ d.sgj[j];
            const uint64_t g = base | dep_tid | d.gj[j];
            float2 a = sm[se], b = sm[se ^ 1u];
            __stcs(reinterpret_cast<VV*>(amps + g), make_float4(a.x, a.y, b.x, b.y));
        }
        __syncthreads();
    }
    // after a timed-out wait, give the outstanding copy and MMAs a bounded chance to land before freeing
    if (c.failed) {
        tc::mbar_wait(&bar, c.parity ^ 1u);
        tc::mbar_wait(&ibar, c.iparity ^ 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid < 32) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(c.tmem), "r"(ncols) : "memory");
    }
}

// ---------------------------------------------------------------------------
// FP16-split tensor-core sweeps (RQ_EXEC_SWEEP_TC16)
// ---------------------------------------------------------------------------
//
// Same tiles, phases and register rows as k_sweep_tc, with the dense 32x32 op
// computed as three FP16 MMA passes, D = Ah*Bh + Ah*Bl + Al*Bh, accumulated in
// FP32 (kind::f16 runs at twice the TF32 rate, and both A parts fit in tensor
// memory at once, so a phase is one MMA round trip instead of two):
//
// * amplitudes are scaled per tile by a power of two 2^s chosen in the tile's
//   first phase from its largest component M: the tile's norm is at most
//   2^(m/2) M, the ops are unitary on the tile, so no component of any phase
//   exceeds that norm, and 2^(m/2) M 2^s <= 2^15 keeps every FP16 high part
//   in range; a small tile gets a large s, so nothing drops into FP16
//   subnormals early;
// * the last phase restores the tile's norm (measured on the scaled inputs in
//   the first phase): the phases are unitary on the tile, and the tensor
//   cores' FP32 accumulation rounds partial sums toward zero, which would
//   otherwise shrink every amplitude by ~1e-7 per phase;
// * a thread's scaled amplitude x splits into h = x rounded to 11 significant
//   bits (exact in FP16) and l = x - h (exact in FP32, then rounded to FP16):
//   the split keeps ~22 bits, and the dropped Al*Bl term is ~2^-22 relative,
//   the same as 3xTF32;
// * the images hold U * 2^14 as FP16 high and low parts (host-built, f64);
//   outputs are scaled back by 2^-14 between phases (the tile stays scaled by
//   2^s) and by 2^-(s+14) in the last phase;
// * tensor memory per 128-row half: accumulator (64 columns), A high part (32
//   columns of FP16 pairs: column i = amplitude i, real part in the low 16
//   bits) and A low part (32 columns);
// * each half is issued by its own thread (warp 4h, lane 0) with its own
//   completion mbarrier, so one half's MMAs overlap the other half's
//   conversion; the CTA meets once per phase (the shared-memory exchange);
// * operand images are double-buffered on 13- and 14-qubit tiles: while a
//   phase's MMAs run, the next phase's image (or the next tile's first image)
//   is already being copied; 12-qubit tiles keep one buffer, so that four CTAs
//   fit on an SM, and copy the next image in once their MMAs are done.
namespace tc16 {

constexpr uint32_t IMG_BYTES = DENSE_F16_WORDS * 4u;   // 16 KB: high + low part
constexpr uint32_t PART_BYTES = IMG_BYTES / 2;
constexpr uint32_t B_SBO = 1024;   // bytes between 8-row groups (8 core matrices along K)
constexpr uint32_t B_LBO = 128;    // bytes between core matrices along K
// FP16 x FP16 -> F32, both operands K-major, M = 128, N = 64
constexpr uint32_t IDESC = (1u << 4) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)(B_LBO >> 4) << 16;
    d |= (uint64_t)(B_SBO >> 4) << 32;
    d |= (uint64_t)1 << 46;   // sm_100 descriptor version; no swizzle, base offset 0
    return d;
}

__device__ __forceinline__ float pow2f(int k) { return __int_as_float((k + 127) << 23); }   // |k| <= 126

__device__ __forceinline__ void st16u(uint32_t taddr, const uint32_t* v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
        ::"r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]),
        "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}

__device__ __forceinline__ void mma(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "r"(a), "l"(bdesc), "r"(IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void start_copy(uint32_t dst, const void* src, uint64_t* bar) {
    const uint32_t b = tc::smem_u32(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(IMG_BYTES) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(IMG_BYTES), "r"(b)
                 : "memory");
}

__device__ __forceinline__ void bar_half(uint32_t half) {   // the 128 threads of one half
    asm volatile("bar.sync %0, 128;" ::"r"(1u + half) : "memory");
}

// index of the lowest set bit of 1 <= g < 32 (the Gray-code bit that flips at step g)
__host__ __device__ constexpr int ctz5(int g) { return (g & 1) ? 0 : (g & 2) ? 1 : (g & 4) ? 2 : (g & 8) ? 3 : 4; }

// packed FP32x2 arithmetic (one instruction for both lanes of a complex value)
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    float2 r;
    asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    float2 r;
    asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    float2 r;
    asm("{.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rc, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}

// bounded wait that lets the thread sleep until the phase completes (or 20 us pass) between
// polls, so waiting warps take no issue slots from the working ones
__device__ __forceinline__ bool wait_sleep(uint64_t* bar, uint32_t parity, uint32_t polls) {
    const uint32_t a = tc::smem_u32(bar);
    for (uint32_t it = 0; it < polls; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity), "r"(20000u)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace tc16

// NTHR = 128: tiles of 12 local qubits, four CTAs per SM, one operand-image buffer (the next
// image is copied in once the CTA's only half has finished its MMAs: a second buffer would
// leave room for three CTAs only, and a fourth independent phase chain per SM hides more of
// the chain's latency than the earlier image copy does); NTHR = 256: 13 local qubits, two
// CTAs per SM; NTHR = 512: 14 local qubits, one CTA (four 128-row halves, all 512
// tensor-memory columns) per SM.  NTHR = 256 and 512 double-buffer the images.
template <int NTHR>
__global__ void __launch_bounds__(NTHR, 512 / NTHR) k_sweep_tc16(float2* __restrict__ amps, const SweepDesc d,
                                                     const PhaseDesc* __restrict__ phases,
                                                     const SwOp* __restrict__ ops,
                                                     const uint32_t* __restrict__ images, uint64_t ntiles) {
    using VV = float4;
    constexpr int NR = 32;
    constexpr bool ONE_BUF = NTHR == 128;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t tile_elems = 1u << d.m;
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    unsigned char* img = reinterpret_cast<unsigned char*>(sm + tile_elems);   // one or two image buffers
    PhaseDesc* sph = reinterpret_cast<PhaseDesc*>(img + (ONE_BUF ? 1u : 2u) * tc16::IMG_BYTES);
    const uint32_t nph = d.phase_end - d.phase_begin;
    const uint32_t op0 = phases[d.phase_begin].op_begin, nops = phases[d.phase_end - 1].op_end - op0;
    SwOp* sop = reinterpret_cast<SwOp*>(sph + nph);
    __shared__ __align__(8) uint64_t mbar[NTHR / 128], ibar[2];
    __shared__ uint32_t tmem_base;
    __shared__ float wmax[NTHR / 32], wsum[NTHR / 32], wsum2[NTHR / 32];
    __shared__ int half_failed[NTHR / 128];

    const uint32_t tid = threadIdx.x;
    const uint32_t T_ = blockDim.x;
    const uint32_t warp = tid >> 5, half = warp >> 2;
    for (uint32_t k = tid; k < nph * (uint32_t)(sizeof(PhaseDesc) / 16); k += T_)
        reinterpret_cast<uint4*>(sph)[k] = reinterpret_cast<const uint4*>(phases + d.phase_begin)[k];
    for (uint32_t k = tid; k < nops; k += T_) sop[k] = ops[op0 + k];
    const uint32_t ncols = 128u * (T_ / 128u);
    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(&tmem_base)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int k = 0; k < NTHR / 128; ++k) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc::smem_u32(&mbar[k])), "r"(1u) : "memory");
            half_failed[k] = 0;
        }
        for (int k = 0; k < 2; ++k)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc::smem_u32(&ibar[k])), "r"(1u) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const PhaseDesc* lph = sph - d.phase_begin;
    const SwOp* lop = sop - op0;
    // each poll may sleep up to 20 us: 2^-7 of the polls of the spinning kernels (~2.6 s in all)
    const uint32_t hpolls = tc::g_tc_wait_polls >> 7;

    const uint64_t cmask = (1ull << d.c) - 1;
    uint64_t dep_tid = 0;
    {
        const uint64_t x = (uint64_t)tid * 2;
        dep_tid = x & cmask;
        for (uint32_t b = d.c; b < d.m; ++b)
            if ((x >> b) & 1ull) dep_tid |= 1ull << d.local_global[b];
    }
    const uint32_t stid = swz16(tid * 2);   // the FP16 kernel's layout (retable_f16)
    auto tile_base = [&](uint64_t tile) {
        uint64_t b = 0;
        for (uint32_t k = 0; k < d.nonlocal_count; ++k)
            if ((tile >> k) & 1ull) b |= 1ull << d.nonlocal[k];
        return b;
    };
    // the operand image of phase p for a tile at `base` (its variant: the tile's values of the
    // phase's qubits outside the tile)
    auto image_of = [&](uint64_t base, uint32_t p) {
        const SwOp& op = lop[lph[p].op_begin];
        uint32_t var = 0;
        for (int j = 0; j < dense_nvq(op); ++j) var |= (uint32_t)((base >> dense_vq(op, j)) & 1ull) << j;
        return images + (size_t)(op.mat + var) * DENSE_F16_WORDS;
    };

    // thread 0 issues every image copy; copies into buffer b complete phases of ibar[b]
    uint32_t issued[2] = {0u, 0u};   // (thread 0) copies issued into each buffer
    uint32_t step = 0;               // (tile, phase) steps run by this CTA
    bool failed = false;
    bool committed = false;          // (issuing threads) MMAs of the current step in flight
    const uint32_t col_h = half * 128u;
    const uint32_t lane_base = ((warp & 3u) * 32u) << 16;

    uint64_t tile = blockIdx.x;
    uint64_t base = tile < ntiles ? tile_base(tile) : 0;
    if (tid == 0 && tile < ntiles) {
        tc16::start_copy(tc::smem_u32(img), image_of(base, d.phase_begin), &ibar[0]);
        issued[0] = 1;
    }
    for (; tile < ntiles && !failed; tile += gridDim.x) {
        const uint64_t next = tile + gridDim.x;
        const uint64_t nbase = next < ntiles ? tile_base(next) : 0;
        issue_tile<float>(sm, amps, d, base, dep_tid, stid);
        cp_async_commit();
        if (next < ntiles) {
            // Pull the next tile into L2 while this one runs its phases: thread t prefetches the
            // t-th contiguous run of 2^c amplitudes (local bits c.. of t << c; 2^(m-c) runs, one
            // per thread), so the next tile's loads hit L2 instead of waiting on HBM.
            uint64_t g = nbase;
            const uint32_t x = tid << d.c;
            for (uint32_t b = d.c; b < d.m; ++b)
                if ((x >> b) & 1u) g |= 1ull << d.local_global[b];
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(amps + g), "r"(8u << d.c) : "memory");
        }
        cp_async_wait0();
        __syncthreads();
        const float mid_scale = tc16::pow2f(-DENSE_F16_SCALE_LOG2);
        float last_scale = 1.f;
        for (uint32_t p = d.phase_begin; p < d.phase_end; ++p, ++step) {
            const uint32_t buf = step & 1u;
            const PhaseDesc& ph = lph[p];
            // the next step's image into the other buffer (its previous MMAs finished last step)
            if (!ONE_BUF && tid == 0) {
                const bool more = p + 1 < d.phase_end;
                if (more || next < ntiles) {
                    tc16::start_copy(tc::smem_u32(img + (buf ^ 1u) * tc16::IMG_BYTES),
                                     more ? image_of(base, p + 1) : image_of(nbase, d.phase_begin), &ibar[buf ^ 1u]);
                    ++issued[buf ^ 1u];
                }
            }
            const bool first = p == d.phase_begin;
            const bool last = p + 1 == d.phase_end;
            // this thread's row: thread bit b sits at local bit tbit_local[b], whose swizzled
            // offset is tsw[b] (the layout is XOR-linear)
            uint32_t sb = 0;
            {
                const uint4 t4 = *reinterpret_cast<const uint4*>(ph.tsw);
                const uint32_t tw[4] = {t4.x, t4.y, t4.z, t4.w};
#pragma unroll
                for (uint32_t b = 0; b < 8; ++b)
                    if ((tid >> b) & 1u) sb ^= (tw[b >> 1] >> (16 * (b & 1u))) & 0xFFFFu;
                if (NTHR > 256 && ((tid >> 8) & 1u)) sb ^= swz16(1u << ph.tbit_local[8]);   // a ninth thread bit
            }
            // register i sits at sb ^ (XOR of S[k] over the set bits k of i); visiting the
            // registers in Gray-code order makes each address one XOR from the previous one
            uint32_t S[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) S[k] = ph.slut[1 << k];
            float2 reg[NR];
            {
                uint32_t a = sb;
#pragma unroll
                for (int g = 0; g < NR; ++g) {
                    if (g) a ^= S[tc16::ctz5(g)];
                    reg[g ^ (g >> 1)] = sm[a];
                }
            }
            if (first) {
                // the tile's largest component M < 2^(E+1) bounds its norm by 2^(m/2) M, and the
                // norm bounds every component of every later phase (unitary on the tile): the
                // scale 2^s with 2^(m/2) M 2^s <= 2^15 keeps all FP16 high parts in range
                float mx = 0.f;
#pragma unroll
                for (int i = 0; i < NR; ++i) mx = fmaxf(mx, fmaxf(fabsf(reg[i].x), fabsf(reg[i].y)));
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
                if ((tid & 31u) == 0) wmax[warp] = mx;
                __syncthreads();
                for (uint32_t w = 0; w < T_ / 32u; ++w) mx = fmaxf(mx, wmax[w]);
                int sc = 0;
                if (mx > 0.f && mx < 3.0e38f) {
                    const int E = (int)((__float_as_uint(mx) >> 23) & 0xFFu) - 127;   // mx in [2^E, 2^(E+1))
                    sc = max(-100, min(100, 14 - E - (int)((d.m + 1) / 2)));
                }
                last_scale = tc16::pow2f(-(sc + DENSE_F16_SCALE_LOG2));
                const float2 s2 = make_float2(tc16::pow2f(sc), tc16::pow2f(sc));
                float2 n2 = make_float2(0.f, 0.f);   // the scaled tile's norm^2, this thread's part
#pragma unroll
                for (int i = 0; i < NR; ++i) {
                    reg[i] = tc16::mul2(reg[i], s2);
                    n2 = tc16::fma2(reg[i], reg[i], n2);
                }
                float n = n2.x + n2.y;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xFFFFFFFFu, n, o);
                if ((tid & 31u) == 0) wsum[warp] = n;   // read at the tile's store, after later CTA barriers
            }
            // A high part h = fp16(x) and low part fp16(x - h) into this thread's tensor-memory lane
            {
                const uint32_t ta = tmem + lane_base + col_h + 64u;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    uint32_t hw[16], lw[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const float2 x = reg[16 * c + j];
                        const __half2 h = __float22half2_rn(x);
                        const __half2 l = __float22half2_rn(tc16::sub2(x, __half22float2(h)));
                        hw[j] = *reinterpret_cast<const uint32_t*>(&h);
                        lw[j] = *reinterpret_cast<const uint32_t*>(&l);
                    }
                    tc16::st16u(ta + 16u * c, hw);
                    tc16::st16u(ta + 32u + 16u * c, lw);
                }
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            }
            tc16::bar_half(half);
            const uint32_t mpar = step & 1u;
            if ((tid & 127u) == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                // with one buffer the n-th copy completes phase n of ibar[0]; with two, copies
                // alternate between the buffers
                const bool landed = ONE_BUF ? tc16::wait_sleep(&ibar[0], step & 1u, hpolls)
                                            : tc16::wait_sleep(&ibar[buf], (step >> 1) & 1u, hpolls);
                if (landed) {
                    const uint32_t bh = tc::smem_u32(img + (ONE_BUF ? 0u : buf) * tc16::IMG_BYTES);
                    const uint32_t bl = bh + tc16::PART_BYTES;
                    const uint32_t dt = tmem + col_h, ah = tmem + col_h + 64u, al = tmem + col_h + 96u;
                    // the small correction products first, then the large one on top of them:
                    // fewer additions into a large running sum, where the accumulator rounds
#pragma unroll
                    for (uint32_t ks = 0; ks < 4; ++ks) tc16::mma(dt, al + 8u * ks, tc16::sdesc(bh + 256u * ks), ks > 0);
#pragma unroll
                    for (uint32_t ks = 0; ks < 4; ++ks) tc16::mma(dt, ah + 8u * ks, tc16::sdesc(bl + 256u * ks), 1u);
#pragma unroll
                    for (uint32_t ks = 0; ks < 4; ++ks) tc16::mma(dt, ah + 8u * ks, tc16::sdesc(bh + 256u * ks), 1u);
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     tc::smem_u32(&mbar[half]))
                                 : "memory");
                    committed = true;
                } else {
                    // the image never landed: release this half's waiters and give up
                    half_failed[half] = 1;
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(&mbar[half])) : "memory");
                }
            }
            if (!tc16::wait_sleep(&mbar[half], mpar, hpolls)) failed = true;
            if (ONE_BUF && tid == 0 && !failed && !half_failed[0]) {
                // the only half's MMAs have read the image: copy in the next step's
                const bool more = p + 1 < d.phase_end;
                if (more || next < ntiles) {
                    tc16::start_copy(tc::smem_u32(img), more ? image_of(base, p + 1) : image_of(nbase, d.phase_begin),
                                     &ibar[0]);
                    ++issued[0];
                }
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (half_failed[half]) failed = true;
            {
                const uint32_t taddr = tmem + lane_base + col_h;
                tc::ld16(taddr, reg);
                tc::ld16(taddr + 16, reg + 8);
                tc::ld16(taddr + 32, reg + 16);
                tc::ld16(taddr + 48, reg + 24);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                if (last) {   // the tile's output norm^2, this thread's part (see the store)
                    float2 o2 = make_float2(0.f, 0.f);
#pragma unroll
                    for (int i = 0; i < NR; ++i) o2 = tc16::fma2(reg[i], reg[i], o2);
                    float o = o2.x + o2.y;
#pragma unroll
                    for (int k = 16; k > 0; k >>= 1) o += __shfl_xor_sync(0xFFFFFFFFu, o, k);
                    if ((tid & 31u) == 0) wsum2[warp] = o;
                }
                const float os = last ? last_scale : mid_scale;
                const float2 os2 = make_float2(os, os);
                uint32_t a = sb;
#pragma unroll
                for (int g = 0; g < NR; ++g) {
                    if (g) a ^= S[tc16::ctz5(g)];
                    sm[a] = tc16::mul2(reg[g ^ (g >> 1)], os2);
                }
            }
            if (__syncthreads_or(failed)) {
                failed = true;
                break;
            }
            committed = false;
        }
        if (failed) break;
        // The phases are unitary on the tile, so its norm is what it was when loaded; the
        // tensor cores' FP32 accumulation rounds partial sums toward zero and would shrink it
        // by ~1e-7 per phase.  The store gives the tile its loaded norm back.
        float fix = 1.f;
        {
            float in2 = 0.f, out2 = 0.f;
            for (uint32_t w = 0; w < T_ / 32u; ++w) {
                in2 += wsum[w];
                out2 += wsum2[w];
            }
            in2 *= (float)(1u << (2 * DENSE_F16_SCALE_LOG2));   // the outputs carry the images' 2^14 too
            if (out2 > 0.f && in2 > 0.f && out2 < 3.0e38f && in2 < 3.0e38f) fix = sqrtf(in2 / out2);
        }
        const float2 fix2 = make_float2(fix, fix);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const uint32_t se = stid ^ d.sgj[j];
            const uint64_t g = base | dep_tid | d.gj[j];
            const float2 a = tc16::mul2(sm[se], fix2), b = tc16::mul2(sm[se ^ 1u], fix2);
            __stcs(reinterpret_cast<VV*>(amps + g), make_float4(a.x, a.y, b.x, b.y));
        }
        __syncthreads();
        base = nbase;
    }
    if (failed) {
        if (tid == 0) tc::g_tc_timeout = 1;
        // let everything still in flight land before the shared and tensor memory are released
        if ((tid & 127u) == 0 && committed) tc::mbar_wait(&mbar[half], step & 1u);
        if (tid == 0)
            for (uint32_t b = 0; b < 2; ++b)
                if (issued[b]) tc::mbar_wait(&ibar[b], (issued[b] - 1u) & 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid < 32) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
}

// Operand images of a tensor-core plan, built on the GPU: one CTA of 32 threads per image, one
// thread per column (the phase's ops applied to e_col in exactly rounded f64, the same
// arithmetic as the host restatement in rq_plan.cuh, so the images are bit-identical).
__global__ void __launch_bounds__(32) k_dense_images(const SwOp* __restrict__ ops, const double* __restrict__ mats,
                                                     const DenseJob* __restrict__ jobs, uint32_t njobs,
                                                     uint32_t* __restrict__ images, int fmt, uint32_t words) {
    double v[64];
    for (uint32_t j = blockIdx.x; j < njobs; j += gridDim.x) {
        const DenseJob jb = jobs[j];
        dense_job_column(jb, ops, mats, (int)threadIdx.x, v);
        dense_image_column(v, (int)threadIdx.x, images + (size_t)jb.slot * words, fmt);
    }
}

// ---------------------------------------------------------------------------
// host planner
// ---------------------------------------------------------------------------

// RUQU_SWEEP_PIPE=1 selects the double-buffered persistent kernel (one CTA per
// SM); the default is the single-buffered kernel with two CTAs per SM.
static bool sweep_pipelined() {
    static const bool on = [] {
        const char* e = std::getenv("RUQU_SWEEP_PIPE");
        return e && e[0] == '1';
    }();
    return on;
}

static bool phase_v1() {
    static const bool on = [] {
        const char* e = std::getenv("RUQU_PHASE_V");
        return e && e[0] == '1';
    }();
    return on;
}

template <typename T>
int launch_sweep(rq_state* s, const SweepDesc& d, const PhaseDesc* ph, const SwOp* ops, const void* mats,
                 uint64_t ntiles, uint32_t rb, size_t smem) {
    using V = typename C2<T>::t;
    unsigned threads = 1u << (d.m - rb);
    int sms = rq::num_sms(s->device);
    if (sweep_pipelined()) {
        auto kp = phase_v1() ? k_sweep_pipe<T, std::is_same<T, float>::value ? 5 : 4, true>
                             : k_sweep_pipe<T, std::is_same<T, float>::value ? 5 : 4, false>;
        const size_t smem2 = 2 * smem;
        RQ_CUDA(cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
        int per_sm = 0;
        RQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kp, (int)threads, smem2));
        if (per_sm >= 1) {
            unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)sms * per_sm);
            kp<<<grid, threads, smem2, s->stream>>>((V*)s->amps, d, ph, ops, (const T*)mats, ntiles);
            RQ_CUDA(cudaGetLastError());
            return RQ_OK;
        }
    }
    auto kern = phase_v1() ? k_sweep<T, std::is_same<T, float>::value ? 5 : 4, true>
                           : k_sweep<T, std::is_same<T, float>::value ? 5 : 4, false>;
    RQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // persistent grid: exactly the CTAs that can be resident at once
    int per_sm = 0;
    RQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)threads, smem));
    if (per_sm < 1) return rq::fail(RQ_ERR_CUDA, "sweep kernel does not fit on an SM");
    unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)sms * per_sm);
    kern<<<grid, threads, smem, s->stream>>>((V*)s->amps, d, ph, ops, (const T*)mats, ntiles);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

}  // namespace

// Prepared gate program: the sweep plan with its device-side tables, or
// (per-gate mode) the gate list.  Executing it launches kernels only.
struct rq_plan {
    uint32_t nq = 0;
    int32_t prec = RQ_F64;
    int device = 0;
    int32_t mode = RQ_EXEC_SWEEP;
    std::vector<rq_gate> gates;          // per-gate mode
    std::vector<SweepDesc> descs;        // sweep mode: one launch each
    unsigned char* dev = nullptr;        // phases | ops | matrices | dense operand images
    size_t off_ph = 0, off_ops = 0, off_mat = 0, off_img = 0;
    int tc_passes = 0;                   // > 0: tensor-core sweeps (3 = 3xTF32, 1 = TF32)
    std::vector<PhaseDesc> host_phases;  // tensor-core sweeps: descriptor sizes per launch
    uint64_t ntiles = 0;
    size_t smem = 0;
    uint32_t rb = 0;
    rq_plan_stats stats{};
    // Rebinding to new gate values with the same structure (kinds and qubits): the planner's
    // decisions depend on the structure only, so the sweeps' local sets and the phase plans
    // are kept; new values re-derive the fused matrices (take_sweep over the same local sets)
    // and, for tensor-core plans, the operand images on the GPU.
    bool rebindable = false;
    uint32_t m = 0, c = 0;
    std::vector<uint64_t> sweep_L;                       // planner's local sets (unpadded)
    std::vector<std::vector<PhasePlan>> phase_plans;     // per sweep
    std::vector<std::vector<uint32_t>> sig;              // per sweep: type | q0 << 8 | q1 << 16 per op
    std::vector<uint32_t> shape;                         // kind | q0 << 8 | q1 << 16 per gate
    int dense_fmt = DENSE_TF32;
    size_t off_pre = 0, off_m64 = 0, off_jobs = 0;       // tensor-core plans: image-building inputs
    uint32_t njobs = 0;
    size_t nmats = 0;                                    // doubles in the matrix table
    mutable cudaEvent_t done = nullptr;                  // after the last launch sequence
    mutable cudaStream_t done_stream = nullptr;
    unsigned char* pin = nullptr;                        // pinned staging of new matrix tables
    size_t pin_cap = 0;
    cudaEvent_t pin_free = nullptr;                      // the last copy out of `pin` has finished
};

namespace rq {

static uint32_t sweep_local_qubits(uint32_t nq, int32_t prec) {
    uint32_t m = prec == RQ_F32 ? 13 : 12;
    if (const char* e = std::getenv("RUQU_SWEEP_LOCAL_QUBITS")) {
        int v = std::atoi(e);
        uint32_t cap = prec == RQ_F32 ? 14 : 13;
        if (v >= 8 && (uint32_t)v <= cap) m = (uint32_t)v;
    }
    return std::min(nq, m);
}

// tc_passes > 0 turns every phase into one dense 32x32 op applied on the tensor cores
// (complex f32 states, m in {12, 13} only); tc_min_ops is kept for the ABI of this helper.
namespace {

uint32_t shape_of(const rq_gate& g) { return (uint32_t)g.kind | ((g.q0 & 0xFFu) << 8) | ((g.q1 & 0xFFu) << 16); }

std::vector<uint32_t> sweep_signature(const Sweep& sw) {
    std::vector<uint32_t> sig;
    sig.reserve(sw.ops.size());
    for (const auto& g : sw.ops) sig.push_back((uint32_t)g.type | ((g.q0 & 0xFFu) << 8) | ((g.q1 & 0xFFu) << 16));
    return sig;
}

// the fused matrix table in the kernels' precision
void narrow_mats(const std::vector<double>& mats, int32_t prec, unsigned char* dst) {
    if (prec == RQ_F32) {
        float* f = reinterpret_cast<float*>(dst);
        for (size_t k = 0; k < mats.size(); ++k) f[k] = (float)mats[k];
    } else {
        std::memcpy(dst, mats.data(), mats.size() * sizeof(double));
    }
}

// the operand images of a tensor-core plan from its ops and f64 matrices (already on the device)
int build_images(const rq_plan* P, cudaStream_t st) {
    if (!P->njobs) return RQ_OK;
    const size_t words = dense_image_words(P->dense_fmt);
    const unsigned grid = (unsigned)std::min<uint32_t>(P->njobs, 65535u);
    k_dense_images<<<grid, 32, 0, st>>>(reinterpret_cast<const SwOp*>(P->dev + P->off_pre),
                                        reinterpret_cast<const double*>(P->dev + P->off_m64),
                                        reinterpret_cast<const DenseJob*>(P->dev + P->off_jobs), P->njobs,
                                        reinterpret_cast<uint32_t*>(P->dev + P->off_img), P->dense_fmt,
                                        (uint32_t)words);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

// Every Unitary1Q matrix of the list unitary to 1e-6 (|U^dagger U - I| entrywise; NaN fails).
// The FP16-split tensor-core sweep bounds a tile's components by its norm when it picks the
// tile's scale and restores that norm at the store, which holds for unitary phases only;
// other lists take the 3xTF32 sweep, whose FP32-range operands need no such bound.
bool all_unitary(const rq_gate* gates, uint64_t n) {
    for (uint64_t k = 0; k < n; ++k) {
        if (gates[k].kind != RQ_GATE_UNITARY1Q) continue;
        const double* m = gates[k].m;   // m00 m01 m10 m11 as (re, im)
        const double c00 = m[0] * m[0] + m[1] * m[1] + m[4] * m[4] + m[5] * m[5];
        const double c11 = m[2] * m[2] + m[3] * m[3] + m[6] * m[6] + m[7] * m[7];
        const double c01r = m[0] * m[2] + m[1] * m[3] + m[4] * m[6] + m[5] * m[7];   // conj(m00) m01 + conj(m10) m11
        const double c01i = m[0] * m[3] - m[1] * m[2] + m[4] * m[7] - m[5] * m[6];
        if (!(std::fabs(c00 - 1.0) <= 1e-6 && std::fabs(c11 - 1.0) <= 1e-6 && std::fabs(c01r) <= 1e-6 &&
              std::fabs(c01i) <= 1e-6))
            return false;
    }
    return true;
}

}  // namespace

int plan_build(const rq_state* s, const rq_gate* gates, uint64_t n, int32_t mode, rq_plan** out, int tc_passes,
               uint32_t tc_min_ops, uint32_t m_override) {
    rq_plan* P = new rq_plan();
    P->nq = s->nq;
    P->prec = s->prec;
    P->device = s->device;
    const uint32_t nq = s->nq;
    const uint32_t rb = s->prec == RQ_F32 ? 5 : 4;
    const uint64_t S = s->bytes();
    for (uint64_t k = 0; k < n; ++k)
        if (gates[k].kind != RQ_GATE_BARRIER) P->shape.push_back(shape_of(gates[k]));
    if (mode == RQ_EXEC_PER_GATE || nq < rb + 2) {
        P->mode = RQ_EXEC_PER_GATE;
        for (uint64_t k = 0; k < n; ++k)
            if (gates[k].kind != RQ_GATE_BARRIER) P->gates.push_back(gates[k]);
        P->stats.gates = P->gates.size();
        P->stats.launches = P->gates.size();
        P->stats.exec_mode = RQ_EXEC_PER_GATE;
        for (auto& g : P->gates) {
            uint64_t b = 2 * S;
            if (g.kind == RQ_GATE_CNOT || g.kind == RQ_GATE_SWAP) b = S;
            else if (g.kind == RQ_GATE_CZ) b = S / 2;
            else if (g.kind == RQ_GATE_Z || g.kind == RQ_GATE_S || g.kind == RQ_GATE_SDG || g.kind == RQ_GATE_T ||
                     g.kind == RQ_GATE_TDG || g.kind == RQ_GATE_PHASE) b = S;
            P->stats.hbm_bytes += b;
        }
        P->rebindable = true;
        *out = P;
        return RQ_OK;
    }
    P->mode = RQ_EXEC_SWEEP;
    uint32_t m = m_override ? std::min(nq, m_override) : sweep_local_qubits(nq, s->prec);
    if (tc_passes == TC_F16 && !all_unitary(gates, n)) tc_passes = 3;
    // the tensor-core sweeps' tile shapes: 12 or 13 local qubits, and 14 for the FP16 sweep only
    // (other 14-qubit requests take 13)
    if (m == 14 && tc_passes != TC_F16) m = 13;
    if (s->prec != RQ_F32 || (m != 12 && m != 13 && !(m == 14 && tc_passes == TC_F16))) tc_passes = 0;
    const uint32_t c = std::min<uint32_t>(m, 5);
    std::vector<PGate> pg;
    std::vector<rq_gate> filtered;
    for (uint64_t k = 0; k < n; ++k)
        if (gates[k].kind != RQ_GATE_BARRIER) filtered.push_back(gates[k]);
    if (!to_pgates(filtered.data(), filtered.size(), pg)) {
        delete P;
        return fail(RQ_ERR_CIRCUIT, "circuit error: only unitary gates can be planned");
    }
    const bool tcp = tc_passes > 0;
    auto sweeps = plan_sweeps(pg, nq, m, c, tcp, tc_passes == TC_F16 ? COST_F16 : COST_TF32);
    for (const auto& sw : sweeps) {   // the structure, before build_program pads the local sets
        P->sweep_L.push_back(sw.L);
        P->sig.push_back(sweep_signature(sw));
    }
    P->m = m;
    P->c = c;

    std::vector<PhaseDesc> phases;
    std::vector<SwOp> ops;
    std::vector<double> mats;
    build_program(sweeps, nq, m, c, rb, s->prec == RQ_F32 ? 2 : 1, P->descs, phases, ops, mats, tcp, nullptr,
                  &P->phase_plans);
    std::vector<uint32_t> images;
    std::vector<DenseJob> jobs;
    std::vector<SwOp> pre_ops;
    uint64_t ndense = 0;
    if (tcp) {
        P->dense_fmt = tc_passes == TC_F16 ? DENSE_F16 : DENSE_TF32;
        // the images are built on the GPU below, from the ops before fusion and their f64 matrices
        if (!fuse_dense(P->descs, phases, ops, mats, images, &ndense, P->dense_fmt, &jobs, &pre_ops, false)) {
            delete P;
            return fail(RQ_ERR_CIRCUIT, "tensor-core plan: a phase touches more than 5 qubits outside the tile");
        }
        for (const auto& ph : phases)
            if (ph.op_end != ph.op_begin + 1 || ops[ph.op_begin].type != OP_DENSE) {
                delete P;
                return fail(RQ_ERR_CIRCUIT, "tensor-core plan: a phase is not one dense op");
            }
        if (tc_passes == TC_F16) retable_f16(P->descs, phases, rb);
        P->tc_passes = tc_passes;
        P->mode = RQ_EXEC_SWEEP_TC;
    }

    const size_t mat_elem = s->prec == RQ_F32 ? sizeof(float) : sizeof(double);
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    P->off_ph = 0;
    P->off_ops = align(P->off_ph + phases.size() * sizeof(PhaseDesc));
    P->off_mat = align(P->off_ops + ops.size() * sizeof(SwOp));
    P->off_img = align(P->off_mat + mats.size() * mat_elem);
    P->off_pre = align(P->off_img + images.size() * sizeof(uint32_t));
    P->off_m64 = align(P->off_pre + pre_ops.size() * sizeof(SwOp));
    P->off_jobs = align(P->off_m64 + (tcp ? mats.size() * sizeof(double) : 0));
    const size_t total = P->off_jobs + jobs.size() * sizeof(DenseJob);
    std::vector<unsigned char> host(total, 0);
    std::memcpy(host.data() + P->off_ph, phases.data(), phases.size() * sizeof(PhaseDesc));
    std::memcpy(host.data() + P->off_ops, ops.data(), ops.size() * sizeof(SwOp));
    narrow_mats(mats, s->prec, host.data() + P->off_mat);
    if (tcp) {
        std::memcpy(host.data() + P->off_pre, pre_ops.data(), pre_ops.size() * sizeof(SwOp));
        std::memcpy(host.data() + P->off_m64, mats.data(), mats.size() * sizeof(double));
        std::memcpy(host.data() + P->off_jobs, jobs.data(), jobs.size() * sizeof(DenseJob));
    }
    P->njobs = (uint32_t)jobs.size();
    P->nmats = mats.size();
    // Upload in stream order on the state's stream: a synchronous copy from pageable memory may
    // return before its DMA lands, and the state's stream (non-blocking) is not ordered after
    // the legacy stream, so the kernels below could otherwise read the tables half-written.
    cudaError_t e = cudaMalloc((void**)&P->dev, total);
    if (e == cudaSuccess) e = cudaMemcpyAsync(P->dev, host.data(), total, cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) {
        if (P->dev) {
            cudaStreamSynchronize(s->stream);
            cudaFree(P->dev);
        }
        delete P;
        return cuda_fail(e, "plan upload");
    }
    int rc = build_images(P, s->stream);
    if (rc == RQ_OK) {
        e = cudaStreamSynchronize(s->stream);   // a plan is complete when it is handed out
        if (e != cudaSuccess) rc = cuda_fail(e, "operand images");
    }
    if (rc != RQ_OK) {
        cudaFree(P->dev);
        delete P;
        return rc;
    }
    P->smem = ((size_t)1 << m) * s->elem_bytes();
    if (tcp) P->host_phases = phases;
    P->ntiles = 1ull << (nq - m);
    P->rb = rb;
    P->rebindable = true;
    P->stats.gates = filtered.size();
    P->stats.sweeps = P->descs.size();
    P->stats.launches = P->descs.size();
    P->stats.phases = phases.size();
    P->stats.ops = ops.size();
    P->stats.dense_ops = ndense;
    P->stats.hbm_bytes = 2 * S * P->descs.size();
    P->stats.exec_mode = !tcp ? RQ_EXEC_SWEEP : tc_passes == TC_F16 ? RQ_EXEC_SWEEP_TC16
                                               : tc_passes == 1 ? RQ_EXEC_SWEEP_TC_FAST : RQ_EXEC_SWEEP_TC;
    P->stats.local_qubits = m;
    *out = P;
    return RQ_OK;
}

bool plan_same_shape(const rq_plan* P, const rq_gate* gates, uint64_t n) {
    uint64_t k = 0;
    for (uint64_t j = 0; j < n; ++j) {
        if (gates[j].kind == RQ_GATE_BARRIER) continue;
        if (k >= P->shape.size() || P->shape[k] != shape_of(gates[j])) return false;
        ++k;
    }
    return k == P->shape.size();
}

// New gate values for a plan of the same gate structure: re-derive each sweep's fused
// matrices from the planner's recorded local sets, check that every sweep takes the same ops,
// and replace the matrix table (and, for tensor-core plans, rebuild the operand images on the
// GPU) in stream order on s's stream.  RQ_ERR_CIRCUIT when the structure does not match (the
// plan is then unchanged).
int plan_rebind(rq_state* s, rq_plan* P, const rq_gate* gates, uint64_t n) {
    if (!P->rebindable || !plan_same_shape(P, gates, n))
        return fail(RQ_ERR_CIRCUIT, "circuit error: the gate list's kinds and qubits differ from the plan's");
    if (P->tc_passes == TC_F16 && !all_unitary(gates, n))
        return fail(RQ_ERR_CIRCUIT, "circuit error: an FP16-split tensor-core plan holds unitary matrices only");
    if (P->mode == RQ_EXEC_PER_GATE) {
        uint64_t k = 0;
        for (uint64_t j = 0; j < n; ++j)
            if (gates[j].kind != RQ_GATE_BARRIER) P->gates[k++] = gates[j];
        return RQ_OK;
    }
    std::vector<rq_gate> filtered;
    filtered.reserve(P->shape.size());
    for (uint64_t j = 0; j < n; ++j)
        if (gates[j].kind != RQ_GATE_BARRIER) filtered.push_back(gates[j]);
    std::vector<PGate> pg;
    if (!to_pgates(filtered.data(), filtered.size(), pg)) return fail(RQ_ERR_CIRCUIT, "circuit error: unplannable gate");
    std::vector<Sweep> sweeps;
    std::vector<char> taken(pg.size(), 0);
    size_t first = 0;
    for (size_t k = 0; k < P->sweep_L.size(); ++k) {
        Sweep sw = take_sweep(pg, taken, first, P->sweep_L[k], P->nq, P->m);
        sw.L = P->sweep_L[k];
        while (first < pg.size() && taken[first]) ++first;
        if (sweep_signature(sw) != P->sig[k]) {
            P->rebindable = false;
            return fail(RQ_ERR_CIRCUIT, "circuit error: the plan's sweeps cannot be re-derived for these gates");
        }
        sweeps.push_back(std::move(sw));
    }
    if (first != pg.size()) {
        P->rebindable = false;
        return fail(RQ_ERR_CIRCUIT, "circuit error: the plan's sweeps cannot be re-derived for these gates");
    }
    std::vector<SweepDesc> descs;
    std::vector<PhaseDesc> phases;
    std::vector<SwOp> ops;
    std::vector<double> mats;
    build_program(sweeps, P->nq, P->m, P->c, P->rb, P->prec == RQ_F32 ? 2 : 1, descs, phases, ops, mats,
                  P->tc_passes > 0, &P->phase_plans, nullptr);
    if (mats.size() != P->nmats) {
        P->rebindable = false;
        return fail(RQ_ERR_CIRCUIT, "circuit error: the plan's matrix table changed shape");
    }
    // stage the new table in pinned memory (once the previous copy out of it has finished), then
    // copy it in stream order after every earlier launch of this plan, on any stream
    const bool tc = P->tc_passes > 0;
    const size_t bytes = mats.size() * (tc || P->prec == RQ_F64 ? sizeof(double) : sizeof(float));
    if (P->pin_free) RQ_CUDA(cudaEventSynchronize(P->pin_free));
    else RQ_CUDA(cudaEventCreateWithFlags(&P->pin_free, cudaEventDisableTiming));
    if (P->pin_cap < bytes) {
        if (P->pin) cudaFreeHost(P->pin);
        P->pin = nullptr;
        P->pin_cap = 0;
        RQ_CUDA(cudaMallocHost((void**)&P->pin, bytes));
        P->pin_cap = bytes;
    }
    if (tc) std::memcpy(P->pin, mats.data(), bytes);
    else narrow_mats(mats, P->prec, P->pin);
    if (P->done && P->done_stream != s->stream) RQ_CUDA(cudaStreamWaitEvent(s->stream, P->done, 0));
    RQ_CUDA(cudaMemcpyAsync(P->dev + (tc ? P->off_m64 : P->off_mat), P->pin, bytes, cudaMemcpyHostToDevice, s->stream));
    RQ_CUDA(cudaEventRecord(P->pin_free, s->stream));
    if (tc) RQ_TRY(build_images(P, s->stream));
    if (!P->done) RQ_CUDA(cudaEventCreateWithFlags(&P->done, cudaEventDisableTiming));
    RQ_CUDA(cudaEventRecord(P->done, s->stream));
    P->done_stream = s->stream;
    return RQ_OK;
}

int apply_one_gate(rq_state* s, const rq_gate& g);   // rq_capi.cu

// ---- autotuner ---------------------------------------------------------------
// For complex f32 states the CUDA-core sweep and the 3xTF32 tensor-core sweep
// agree to FP32 accuracy, and which is faster depends on the circuit (how many
// gates each phase's dense op absorbs) and the state size.  RQ_EXEC_AUTO times
// both plans on a scratch state of the same shape the first time a gate
// structure (kinds and qubits, not angles) is seen on a device and keeps the
// faster; the choice is cached per (device, qubits, structure).
namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, uint32_t, uint64_t>, std::pair<int, uint32_t>> g_tune;

uint64_t structure_hash(const rq_gate* g, uint64_t n) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        h ^= v;
        h *= 1099511628211ull;
    };
    for (uint64_t k = 0; k < n; ++k) {
        mix((uint64_t)g[k].kind);
        mix((uint64_t)g[k].q0);
        mix((uint64_t)g[k].q1);
    }
    mix(n);
    return h;
}

// device time of one execution of P on a scratch state shaped like t (after one warm-up run)
int time_plan(const rq_state& t, const rq_plan* P, float* ms) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    RQ_CUDA(cudaEventCreate(&e0));
    RQ_CUDA(cudaEventCreate(&e1));
    rq_state u = t;
    int rc = plan_launch(&u, P);
    if (rc == RQ_OK) {
        cudaEventRecord(e0, t.stream);
        rc = plan_launch(&u, P);
        cudaEventRecord(e1, t.stream);
    }
    cudaError_t e = cudaEventSynchronize(e1);
    if (rc == RQ_OK && e != cudaSuccess) rc = cuda_fail(e, "autotune timing");
    if (rc == RQ_OK) cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}
}  // namespace

int autotune_tc(const rq_state* s, const rq_gate* gates, uint64_t n, int* passes, uint32_t* m_out) {
    *passes = 0;
    *m_out = 0;
    const uint32_t m = sweep_local_qubits(s->nq, s->prec);
    if (s->prec != RQ_F32 || (m != 12 && m != 13) || n == 0) return RQ_OK;
    if (const char* e = std::getenv("RUQU_AUTOTUNE"))
        if (e[0] == '0') return RQ_OK;
    const auto key = std::make_tuple(s->device, s->nq, structure_hash(gates, n));
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            *passes = it->second.first;
            *m_out = it->second.second;
            return RQ_OK;
        }
    }
    // candidates: CUDA-core sweep; 3xTF32 and FP16-split tensor-core sweeps with the default
    // tile and with one local qubit fewer (twice the CTAs per SM, more sweeps); the FP16 sweep
    // also with one local qubit more (one 512-thread CTA per SM, fewer sweeps)
    struct Cand {
        int passes;
        uint32_t m;
        rq_plan* plan;
        float ms;
    };
    std::vector<Cand> cands = {{0, 0, nullptr, 0.f}, {3, 0, nullptr, 0.f}, {TC_F16, 0, nullptr, 0.f}};
    if (m == 13 && s->nq > 13) {
        cands.push_back({3, 12, nullptr, 0.f});
        cands.push_back({TC_F16, 12, nullptr, 0.f});
        if (s->nq > 14) cands.push_back({TC_F16, 14, nullptr, 0.f});
    }
    for (auto& c : cands)
        if (plan_build(s, gates, n, RQ_EXEC_SWEEP, &c.plan, c.passes, 2, c.m) != RQ_OK) {
            if (c.passes == 0) {   // the CUDA-core plan is the reference point
                for (auto& d : cands) plan_free(d.plan);
                return fail(RQ_ERR_CIRCUIT, "circuit error: the gate list cannot be planned");
            }
            c.plan = nullptr;       // a circuit the tensor-core planner cannot take
            cudaGetLastError();
        }
    int rc = RQ_OK;
    int best = 0;
    void* scratch = nullptr;
    const bool any_tc = std::any_of(cands.begin() + 1, cands.end(), [](const Cand& c) {
        return c.plan && c.plan->stats.dense_ops > 0;
    });
    if (any_tc && cudaMalloc(&scratch, s->bytes()) == cudaSuccess) {
        rq_state t = *s;
        t.amps = scratch;
        // |0...0>: the circuit's first layers spread it into a dense state, so the candidates are
        // timed on live amplitudes (an all-zero state stays zero and draws less power, which
        // favoured the plans with more HBM passes)
        cudaMemsetAsync(scratch, 0, s->bytes(), s->stream);
        const float one[2] = {1.f, 0.f};   // complex f32 amplitude 0 (pageable: staged before the call returns)
        cudaMemcpyAsync(scratch, one, sizeof(one), cudaMemcpyHostToDevice, s->stream);
        for (size_t k = 0; k < cands.size() && rc == RQ_OK; ++k)
            if (cands[k].plan) rc = time_plan(t, cands[k].plan, &cands[k].ms);
        // a later candidate must be more than 2 % faster than the best so far: near-equal plans
        // (the 12- and 13-qubit FP16 plans of a 30-qubit random-layer circuit are within 1 %)
        // then keep the earlier one, which has fewer sweeps, instead of following timing noise
        if (rc == RQ_OK) {
            float ms[8];
            bool ok[8];
            const size_t nc = std::min<size_t>(cands.size(), 8);   // at most six candidates
            for (size_t k = 0; k < nc; ++k) {
                ms[k] = cands[k].ms;
                ok[k] = cands[k].plan && cands[k].plan->stats.dense_ops > 0;
            }
            best = (int)pick_fastest(ms, ok, nc);
        }
        cudaFree(scratch);
    } else {
        cudaGetLastError();   // no room for a scratch state (or nothing to compare): CUDA-core sweep
    }
    const int choice_passes = cands[best].passes;
    const uint32_t choice_m = cands[best].m;
    for (auto& c : cands) plan_free(c.plan);
    RQ_TRY(rc);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = std::make_pair(choice_passes, choice_m);
    *passes = choice_passes;
    *m_out = choice_m;
    return RQ_OK;
}

// FP16-split tensor-core sweeps: shared memory = tile | two operand images | the sweep's
// phase and op descriptors; resident CTAs per SM by registers (128 per thread), shared
// memory (228 KB per SM, 1 KB reserved per CTA) and tensor memory (512 columns per SM).
static int launch_tc16(rq_state* s, const rq_plan* P, const PhaseDesc* ph, const SwOp* op) {
    const uint32_t* img = reinterpret_cast<const uint32_t*>(P->dev + P->off_img);
    const unsigned threads = 1u << (P->descs.front().m - 5);
    const PhaseDesc* hph = P->host_phases.data();
    auto smem_of = [&](const SweepDesc& d) {
        const size_t nph = d.phase_end - d.phase_begin;
        const size_t nops = hph[d.phase_end - 1].op_end - hph[d.phase_begin].op_begin;
        return P->smem + (threads == 128 ? 1u : 2u) * (size_t)tc16::IMG_BYTES + nph * sizeof(PhaseDesc) +
               nops * sizeof(SwOp);
    };
    size_t smem_max = 0;
    for (const auto& d : P->descs) smem_max = std::max(smem_max, smem_of(d));
    const int by_regs = 65536 / (128 * (int)threads);
    const int by_smem = (int)((228u * 1024u) / (smem_max + 1024u + 128u));
    const int by_tmem = (int)(512u / (128u * (threads / 128u)));
    const int per_sm = std::min(by_regs, std::min(by_smem, by_tmem));
    if (per_sm < 1) return fail(RQ_ERR_CUDA, "FP16 tensor-core sweep kernel does not fit on an SM");
    const unsigned grid = (unsigned)std::min<uint64_t>(P->ntiles, (uint64_t)per_sm * rq::num_sms(s->device));
    for (const auto& d : P->descs) {
        const size_t smem = smem_of(d);
        auto kern = threads > 256 ? k_sweep_tc16<512> : threads > 128 ? k_sweep_tc16<256> : k_sweep_tc16<128>;
        RQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, threads, smem, s->stream>>>((float2*)s->amps, d, ph, op, img, P->ntiles);
        RQ_CUDA(cudaGetLastError());
    }
    return RQ_OK;
}

static int plan_launch_kernels(rq_state* s, const rq_plan* P);

// Launch a prepared plan on s's stream; the plan remembers the stream and an event after the
// launches, so that new matrix tables (plan_rebind) are written only once they have run.
int plan_launch(rq_state* s, const rq_plan* P) {
    // the plan's last use (launches or new tables) on another stream comes first
    if (P->done && P->done_stream != s->stream) RQ_CUDA(cudaStreamWaitEvent(s->stream, P->done, 0));
    RQ_TRY(plan_launch_kernels(s, P));
    if (P->mode != RQ_EXEC_PER_GATE) {
        if (!P->done) RQ_CUDA(cudaEventCreateWithFlags(&P->done, cudaEventDisableTiming));
        RQ_CUDA(cudaEventRecord(P->done, s->stream));
        P->done_stream = s->stream;
    }
    return RQ_OK;
}

static int plan_launch_kernels(rq_state* s, const rq_plan* P) {
    if (P->mode == RQ_EXEC_PER_GATE) {
        for (const auto& g : P->gates) RQ_TRY(apply_one_gate(s, g));
        return RQ_OK;
    }
    const PhaseDesc* ph = reinterpret_cast<const PhaseDesc*>(P->dev + P->off_ph);
    const SwOp* op = reinterpret_cast<const SwOp*>(P->dev + P->off_ops);
    const void* mt = P->dev + P->off_mat;
    if (P->tc_passes == TC_F16) return launch_tc16(s, P, ph, op);
    if (P->tc_passes > 0) {
        const float* img = reinterpret_cast<const float*>(P->dev + P->off_img);
        const size_t img_bytes = (P->tc_passes > 1 ? DENSE_IMAGE_FLOATS : DENSE_FLOATS) * sizeof(float);
        const unsigned threads = 1u << (P->descs.front().m - 5);
        // resident CTAs per SM: by registers and shared memory, and by tensor memory (512 columns per SM)
        size_t smem_max = 0;
        for (const auto& d : P->descs) {
            const size_t nph = d.phase_end - d.phase_begin;
            const size_t nops = P->host_phases[d.phase_end - 1].op_end - P->host_phases[d.phase_begin].op_begin;
            smem_max = std::max(smem_max, P->smem + img_bytes + nph * sizeof(PhaseDesc) + nops * sizeof(SwOp));
        }
        // 128 registers per thread (launch bounds), 228 KB of shared memory per SM (1 KB reserved per CTA)
        const int by_regs = 65536 / (128 * (int)threads);
        const int by_smem = (int)((228u * 1024u) / (smem_max + 1024u + 64u));
        const int by_tmem = (int)(512u / (128u * (threads / 128u)));
        int per_sm = std::min(by_regs, std::min(by_smem, by_tmem));
        if (per_sm < 1) return fail(RQ_ERR_CUDA, "tensor-core sweep kernel does not fit on an SM");
        const unsigned grid = (unsigned)std::min<uint64_t>(P->ntiles, (uint64_t)per_sm * rq::num_sms(s->device));
        const PhaseDesc* hph = P->host_phases.data();
        for (const auto& d : P->descs) {
            const size_t nph = d.phase_end - d.phase_begin;
            const size_t nops = hph[d.phase_end - 1].op_end - hph[d.phase_begin].op_begin;
            const size_t smem = P->smem + img_bytes + nph * sizeof(PhaseDesc) + nops * sizeof(SwOp);
            RQ_CUDA(cudaFuncSetAttribute(k_sweep_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_sweep_tc<<<grid, threads, smem, s->stream>>>((float2*)s->amps, d, ph, op, (const float*)mt, img,
                                                          P->ntiles, P->tc_passes);
            RQ_CUDA(cudaGetLastError());
        }
        return RQ_OK;
    }
    for (const auto& d : P->descs) {
        if (s->prec == RQ_F32) RQ_TRY(launch_sweep<float>(s, d, ph, op, mt, P->ntiles, P->rb, P->smem));
        else RQ_TRY(launch_sweep<double>(s, d, ph, op, mt, P->ntiles, P->rb, P->smem));
    }
    return RQ_OK;
}

void plan_free(rq_plan* P) {
    if (!P) return;
    cudaSetDevice(P->device);
    // the plan's last launches and table copies may still be running on another state's
    // stream: let them finish before the device tables and the pinned staging are released
    if (P->done) cudaEventSynchronize(P->done);
    if (P->pin_free) cudaEventSynchronize(P->pin_free);
    if (P->dev) cudaFree(P->dev);
    if (P->pin) cudaFreeHost(P->pin);
    if (P->pin_free) cudaEventDestroy(P->pin_free);
    if (P->done) cudaEventDestroy(P->done);
    delete P;
}

rq_plan_stats plan_stats(const rq_plan* p) { return p->stats; }

int tc_timeout_flag(int* out) {
    int v = 0, zero = 0;
    RQ_CUDA(cudaMemcpyFromSymbol(&v, tc::g_tc_timeout, sizeof(int)));
    if (v) {
        RQ_CUDA(cudaMemcpyToSymbol(tc::g_tc_timeout, &zero, sizeof(int)));
        RQ_CUDA(cudaDeviceSynchronize());
    }
    *out = v;
    return RQ_OK;
}

int sync_checked(rq_state* s) {
    RQ_CUDA(cudaStreamSynchronize(s->stream));
    int to = 0;
    RQ_TRY(tc_timeout_flag(&to));
    if (to) return fail(RQ_ERR_TIMEOUT, "a tensor-core sweep's bounded device wait expired; the state is invalid");
    return RQ_OK;
}

int tc_set_wait_polls(uint32_t polls) {
    const uint32_t v = polls == RQ_WAIT_LIMIT_DEFAULT ? tc::WAIT_POLLS : polls;
    RQ_CUDA(cudaMemcpyToSymbol(tc::g_tc_wait_polls, &v, sizeof(v)));
    RQ_CUDA(cudaDeviceSynchronize());   // landed before any later launch, on any stream
    return RQ_OK;
}

bool plan_fits(const rq_plan* p, const rq_state* s) {
    return p->nq == s->nq && p->prec == s->prec && p->device == s->device;
}

// Prepared programs of recent gate lists, so that applying the same list again (a circuit
// re-run from |0>, the repeated evaluations of a driver) skips the host planning and the
// upload.  Keyed by device, qubit count, precision, tensor-core passes and every byte of
// the gate list; a few entries, oldest evicted (its cudaFree waits for launches reading it).
namespace {
struct CachedPlan {
    int device;
    uint32_t nq;
    int32_t prec;
    int passes;
    uint32_t m;
    uint64_t hash;
    std::vector<rq_gate> gates;
    rq_plan* plan;
};
std::mutex g_plan_mu;
std::vector<CachedPlan> g_plans;
constexpr size_t PLAN_CACHE = 4;

uint64_t bytes_hash(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    uint64_t h = 1469598103934665603ull;
    for (size_t k = 0; k < n; ++k) {
        h ^= b[k];
        h *= 1099511628211ull;
    }
    return h;
}
}  // namespace

int apply_sweeps(rq_state* s, const rq_gate* gates, uint64_t n, int tc_passes, uint32_t m) {
    if (n == 0) return RQ_OK;
    const uint64_t h = bytes_hash(gates, n * sizeof(rq_gate));
    std::lock_guard<std::mutex> lk(g_plan_mu);
    for (size_t k = 0; k < g_plans.size(); ++k) {
        CachedPlan& c = g_plans[k];
        if (c.device == s->device && c.nq == s->nq && c.prec == s->prec && c.passes == tc_passes && c.m == m &&
            c.hash == h &&
            c.gates.size() == n && std::memcmp(c.gates.data(), gates, n * sizeof(rq_gate)) == 0) {
            std::rotate(g_plans.begin() + k, g_plans.begin() + k + 1, g_plans.end());   // most recent last
            return plan_launch(s, g_plans.back().plan);
        }
    }
    // the same gate structure with other angles (a driver's next evaluation): new matrix tables
    // and operand images for the cached plan, no planning
    for (size_t k = g_plans.size(); k-- > 0;) {
        CachedPlan& c = g_plans[k];
        if (c.device == s->device && c.nq == s->nq && c.prec == s->prec && c.passes == tc_passes && c.m == m &&
            c.gates.size() == n && c.plan->rebindable && plan_same_shape(c.plan, gates, n)) {
            if (plan_rebind(s, c.plan, gates, n) != RQ_OK) break;   // not re-derivable: plan afresh below
            c.gates.assign(gates, gates + n);
            c.hash = h;
            std::rotate(g_plans.begin() + k, g_plans.begin() + k + 1, g_plans.end());
            return plan_launch(s, g_plans.back().plan);
        }
    }
    rq_plan* P = nullptr;
    RQ_TRY(plan_build(s, gates, n, RQ_EXEC_SWEEP, &P, tc_passes, 2, m));
    int rc = plan_launch(s, P);
    if (rc != RQ_OK) {
        plan_free(P);
        return rc;
    }
    if (g_plans.size() >= PLAN_CACHE) {
        cudaSetDevice(g_plans.front().device);
        plan_free(g_plans.front().plan);
        g_plans.erase(g_plans.begin());
        cudaSetDevice(s->device);
    }
    g_plans.push_back(CachedPlan{s->device, s->nq, s->prec, tc_passes, m, h, std::vector<rq_gate>(gates, gates + n), P});
    return RQ_OK;
}

}  // namespace rq
