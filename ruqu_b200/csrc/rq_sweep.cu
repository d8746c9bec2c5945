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

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>
#include <cstdlib>

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

template <typename T, int RB>
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
    const uint32_t T_ = blockDim.x;
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
        run_phases<T, RB>(sm, d, phases, ops, mats, base, tid);

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
template <typename T, int RB>
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
        run_phases<T, RB>(sm, d, phases, ops, mats, base, tid);
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
// host planner
// ---------------------------------------------------------------------------

// Double-buffered persistent sweeps (default); RUQU_SWEEP_PIPE=0 selects the
// single-buffered kernel with two CTAs per SM.
static bool sweep_pipelined() {
    static const bool on = [] {
        const char* e = std::getenv("RUQU_SWEEP_PIPE");
        return !(e && e[0] == '0');
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
        auto kp = k_sweep_pipe<T, std::is_same<T, float>::value ? 5 : 4>;
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
    auto kern = k_sweep<T, std::is_same<T, float>::value ? 5 : 4>;
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
    unsigned char* dev = nullptr;        // phases | ops | matrices
    size_t off_ph = 0, off_ops = 0, off_mat = 0;
    uint64_t ntiles = 0;
    size_t smem = 0;
    uint32_t rb = 0;
    rq_plan_stats stats{};
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

int plan_build(const rq_state* s, const rq_gate* gates, uint64_t n, int32_t mode, rq_plan** out) {
    rq_plan* P = new rq_plan();
    P->nq = s->nq;
    P->prec = s->prec;
    P->device = s->device;
    const uint32_t nq = s->nq;
    const uint32_t rb = s->prec == RQ_F32 ? 5 : 4;
    const uint64_t S = s->bytes();
    if (mode == RQ_EXEC_PER_GATE || nq < rb + 2) {
        P->mode = RQ_EXEC_PER_GATE;
        for (uint64_t k = 0; k < n; ++k)
            if (gates[k].kind != RQ_GATE_BARRIER) P->gates.push_back(gates[k]);
        P->stats.gates = P->gates.size();
        P->stats.launches = P->gates.size();
        for (auto& g : P->gates) {
            uint64_t b = 2 * S;
            if (g.kind == RQ_GATE_CNOT || g.kind == RQ_GATE_SWAP) b = S;
            else if (g.kind == RQ_GATE_CZ) b = S / 2;
            else if (g.kind == RQ_GATE_Z || g.kind == RQ_GATE_S || g.kind == RQ_GATE_SDG || g.kind == RQ_GATE_T ||
                     g.kind == RQ_GATE_TDG || g.kind == RQ_GATE_PHASE) b = S;
            P->stats.hbm_bytes += b;
        }
        *out = P;
        return RQ_OK;
    }
    P->mode = RQ_EXEC_SWEEP;
    const uint32_t m = sweep_local_qubits(nq, s->prec);
    const uint32_t c = std::min<uint32_t>(m, 5);
    std::vector<PGate> pg;
    std::vector<rq_gate> filtered;
    for (uint64_t k = 0; k < n; ++k)
        if (gates[k].kind != RQ_GATE_BARRIER) filtered.push_back(gates[k]);
    if (!to_pgates(filtered.data(), filtered.size(), pg)) {
        delete P;
        return fail(RQ_ERR_CIRCUIT, "circuit error: only unitary gates can be planned");
    }
    auto sweeps = plan_sweeps(pg, nq, m, c);

    std::vector<PhaseDesc> phases;
    std::vector<SwOp> ops;
    std::vector<double> mats;
    build_program(sweeps, nq, m, c, rb, s->prec == RQ_F32 ? 2 : 1, P->descs, phases, ops, mats);

    size_t mat_elem = s->prec == RQ_F32 ? sizeof(float) : sizeof(double);
    P->off_ph = 0;
    P->off_ops = (P->off_ph + phases.size() * sizeof(PhaseDesc) + 255) & ~size_t(255);
    P->off_mat = (P->off_ops + ops.size() * sizeof(SwOp) + 255) & ~size_t(255);
    size_t total = P->off_mat + mats.size() * mat_elem;
    std::vector<unsigned char> host(total);
    std::memcpy(host.data() + P->off_ph, phases.data(), phases.size() * sizeof(PhaseDesc));
    std::memcpy(host.data() + P->off_ops, ops.data(), ops.size() * sizeof(SwOp));
    if (s->prec == RQ_F32) {
        float* f = reinterpret_cast<float*>(host.data() + P->off_mat);
        for (size_t k = 0; k < mats.size(); ++k) f[k] = (float)mats[k];
    } else {
        std::memcpy(host.data() + P->off_mat, mats.data(), mats.size() * sizeof(double));
    }
    cudaError_t e = cudaMalloc((void**)&P->dev, total);
    if (e == cudaSuccess) e = cudaMemcpy(P->dev, host.data(), total, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        if (P->dev) cudaFree(P->dev);
        delete P;
        return cuda_fail(e, "plan upload");
    }
    P->smem = ((size_t)1 << m) * s->elem_bytes();
    P->ntiles = 1ull << (nq - m);
    P->rb = rb;
    P->stats.gates = filtered.size();
    P->stats.sweeps = P->descs.size();
    P->stats.launches = P->descs.size();
    P->stats.phases = phases.size();
    P->stats.ops = ops.size();
    P->stats.hbm_bytes = 2 * S * P->descs.size();
    *out = P;
    return RQ_OK;
}

int apply_one_gate(rq_state* s, const rq_gate& g);   // rq_capi.cu

int plan_launch(rq_state* s, const rq_plan* P) {
    if (P->mode == RQ_EXEC_PER_GATE) {
        for (const auto& g : P->gates) RQ_TRY(apply_one_gate(s, g));
        return RQ_OK;
    }
    const PhaseDesc* ph = reinterpret_cast<const PhaseDesc*>(P->dev + P->off_ph);
    const SwOp* op = reinterpret_cast<const SwOp*>(P->dev + P->off_ops);
    const void* mt = P->dev + P->off_mat;
    for (const auto& d : P->descs) {
        if (s->prec == RQ_F32) RQ_TRY(launch_sweep<float>(s, d, ph, op, mt, P->ntiles, P->rb, P->smem));
        else RQ_TRY(launch_sweep<double>(s, d, ph, op, mt, P->ntiles, P->rb, P->smem));
    }
    return RQ_OK;
}

void plan_free(rq_plan* P) {
    if (!P) return;
    if (P->dev) {
        cudaSetDevice(P->device);
        cudaFree(P->dev);
    }
    delete P;
}

rq_plan_stats plan_stats(const rq_plan* p) { return p->stats; }

bool plan_fits(const rq_plan* p, const rq_state* s) {
    return p->nq == s->nq && p->prec == s->prec && p->device == s->device;
}

int apply_sweeps(rq_state* s, const rq_gate* gates, uint64_t n) {
    if (n == 0) return RQ_OK;
    rq_plan* P = nullptr;
    RQ_TRY(plan_build(s, gates, n, RQ_EXEC_SWEEP, &P));
    int rc = plan_launch(s, P);
    // cudaFree of the program waits for the launches that read it
    plan_free(P);
    return rc;
}

}  // namespace rq
