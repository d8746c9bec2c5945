// rq_reduce.cu -- FP64-accumulated reductions over the state.
//
// Counterparts of probabilities / probability_of_qubit (state.rs:123-137),
// expectation_value / expectation_hamiltonian (state.rs:362-408), normalize
// and fidelity (state.rs:415-435).  Every reduction accumulates in FP64 (also
// for f32 states) and is deterministic: a fixed grid writes one partial per
// block and term, and a second kernel sums the partials in a fixed order.
#include "rq_internal.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace {

using rqd::C2;
using rqd::insert0;

constexpr int TPB = 256;
constexpr int KMAX = 8;   // Pauli strings per pass

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// sum `v` over the block; result valid in thread 0
__device__ __forceinline__ double block_sum(double v, double* sh) {
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

template <typename V>
__device__ __forceinline__ double norm2(V x) {
    double re = (double)x.x, im = (double)x.y;
    return re * re + im * im;
}

// sum of |a_i|^2 over i with bit q == want (q = 64: all i)
template <typename T>
__global__ void k_prob(const typename C2<T>::t* __restrict__ a, uint64_t count, uint32_t q, int want,
                       double* __restrict__ partials) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < count;
         p += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i = q < 64 ? (insert0(p, q) | ((uint64_t)want << q)) : p;
        acc += norm2(a[i]);
    }
    double r = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

struct TermChunk {
    uint64_t pmask[KMAX];
    int odd[KMAX];
    int k;
};

// Pauli strings sharing one xmask.  x == 0: acc_k += s_k(i)|a_i|^2.
// x != 0: pairs (i, j = i^x) with the top bit h of x clear in i,
// z = conj(a_j) a_i, acc_k += s_k(i) * (odd_k ? Im z : Re z).
template <typename T>
__global__ void k_pauli(const typename C2<T>::t* __restrict__ a, uint64_t count, uint64_t x, uint32_t h,
                        TermChunk tc, double* __restrict__ partials, uint32_t slot0, uint32_t stride) {
    __shared__ double sh[32];
    double acc[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) acc[k] = 0.0;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < count;
         p += (uint64_t)gridDim.x * blockDim.x) {
        double re, im;
        uint64_t i;
        if (x == 0) {
            i = p;
            re = norm2(a[i]);
            im = 0.0;
        } else {
            i = insert0(p, h);
            auto ai = a[i];
            auto aj = a[i ^ x];
            double air = ai.x, aii = ai.y, ajr = aj.x, aji = aj.y;
            re = ajr * air + aji * aii;
            im = ajr * aii - aji * air;
        }
#pragma unroll
        for (int k = 0; k < KMAX; ++k) {
            if (k < tc.k) {
                double v = tc.odd[k] ? im : re;
                acc[k] += (__popcll(i & tc.pmask[k]) & 1) ? -v : v;
            }
        }
    }
    for (int k = 0; k < tc.k; ++k) {
        double r = block_sum(acc[k], sh);
        if (threadIdx.x == 0) partials[(size_t)(slot0 + k) * stride + blockIdx.x] = r;
    }
}

// Single-qubit Z strings (and the identity) in one pass: <Z_q> = sum_x p(x)(1 - 2 bit_q(x)).
// Each thread owns chunks of 32 consecutive amplitudes: per chunk it forms the total
// probability and the five sums over the amplitudes whose low index bit b is set;
// a string on a low qubit (q < 5) adds total - 2 s_q, one on a high qubit adds
// +-total by bit q of the chunk's index, the identity adds total.  Up to ZMAX
// strings per pass; FP64 accumulation, fixed-order block and grid reductions.
constexpr int ZMAX = 32;
struct ZChunk {
    uint8_t q[ZMAX];   // qubit of the string, 64 = identity
    int k;
};

template <typename T> struct ZVec;
template <> struct ZVec<float> { using t = float4; static constexpr int EPV = 2; };
template <> struct ZVec<double> { using t = double2; static constexpr int EPV = 1; };

// Warp-cooperative: warp w of the grid owns segments of 1024 consecutive amplitudes;
// in each, lane l loads the 16-byte vectors it*32 + l (coalesced), so the low index bits
// of every element it sees are fixed by (lane, position in the vector) and the next bits
// by the unrolled `it`: the lane keeps its total, the sum with index bit 0 set (f32) and
// the sums by the bits of `it`; a string's value per segment follows from those
// (bits 0..9) or from the segment index (bits >= 10).
template <typename T>
__global__ void __launch_bounds__(256, 2) k_zsingle(const typename C2<T>::t* __restrict__ a, uint64_t nseg,
                                                    ZChunk zc, double* __restrict__ partials, uint32_t slot0,
                                                    uint32_t stride) {
    using VV = typename ZVec<T>::t;
    constexpr int EPV = ZVec<T>::EPV;
    constexpr int NIT = 1024 / (32 * EPV);    // vectors per lane per segment: 16 (f32) or 32 (f64)
    constexpr int LB = EPV == 2 ? 1 : 0;      // element bits below the lane bits
    constexpr int ITB = EPV == 2 ? 4 : 5;     // bits of `it`
    __shared__ double sh[32];
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    double acc[ZMAX];
#pragma unroll
    for (int k = 0; k < ZMAX; ++k) acc[k] = 0.0;
    for (uint64_t sg = warp; sg < nseg; sg += nwarps) {
        const VV* src = reinterpret_cast<const VV*>(a + sg * 1024);
        double tot = 0.0, odd = 0.0, r[ITB];
#pragma unroll
        for (int k = 0; k < ITB; ++k) r[k] = 0.0;
#pragma unroll
        for (int h = 0; h < NIT; h += 8) {
            VV v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = __ldcs(src + (h + u) * 32 + lane);
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int it = h + u;
                double pit;
                if constexpr (EPV == 2) {
                    const double p0 = (double)v[u].x * v[u].x + (double)v[u].y * v[u].y;
                    const double p1 = (double)v[u].z * v[u].z + (double)v[u].w * v[u].w;
                    odd += p1;
                    pit = p0 + p1;
                } else {
                    pit = (double)v[u].x * v[u].x + (double)v[u].y * v[u].y;
                }
                tot += pit;
#pragma unroll
                for (int k = 0; k < ITB; ++k)
                    if ((it >> k) & 1) r[k] += pit;
            }
        }
        // element index bits inside the segment: [0, LB) vector slot, [LB, LB + 5) lane, then `it`
#pragma unroll
        for (int k = 0; k < ZMAX; ++k) {
            if (k < zc.k) {
                const uint32_t q = zc.q[k];
                double v;
                if (q >= 64) {
                    v = tot;
                } else if (q < (uint32_t)LB) {
                    v = tot - 2.0 * odd;
                } else if (q < (uint32_t)LB + 5) {
                    v = ((lane >> (q - LB)) & 1u) ? -tot : tot;
                } else if (q < 10) {
                    const uint32_t kb = q - LB - 5;
                    double s = r[0];
#pragma unroll
                    for (int t = 1; t < ITB; ++t)
                        if (kb == (uint32_t)t) s = r[t];
                    v = tot - 2.0 * s;
                } else {
                    v = ((sg >> (q - 10)) & 1ull) ? -tot : tot;
                }
                acc[k] += v;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < ZMAX; ++k) {
        if (k < zc.k) {
            double rr = block_sum(acc[k], sh);
            if (threadIdx.x == 0) partials[(size_t)(slot0 + k) * stride + blockIdx.x] = rr;
        }
    }
}

// <a|b> = sum conj(a_i) b_i
template <typename TA, typename TB>
__global__ void k_inner(const typename C2<TA>::t* __restrict__ a, const typename C2<TB>::t* __restrict__ b,
                        uint64_t n, double* __restrict__ partials, uint32_t stride) {
    __shared__ double sh[32];
    double re = 0.0, im = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        auto x = a[i];
        auto y = b[i];
        double xr = x.x, xi = x.y, yr = y.x, yi = y.y;
        re += xr * yr + xi * yi;
        im += xr * yi - xi * yr;
    }
    double r = block_sum(re, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = r;
    r = block_sum(im, sh);
    if (threadIdx.x == 0) partials[stride + blockIdx.x] = r;
}

// out[k] = sum_b partials[k*stride + b], fixed order
__global__ void k_finalize(const double* __restrict__ partials, uint32_t nblocks, uint32_t stride,
                           double* __restrict__ out) {
    __shared__ double sh[32];
    const double* p = partials + (size_t)blockIdx.x * stride;
    double acc = 0.0;
    for (uint32_t b = threadIdx.x; b < nblocks; b += blockDim.x) acc += p[b];
    double r = block_sum(acc, sh);
    if (threadIdx.x == 0) out[blockIdx.x] = r;
}

// p_i = re*re + im*im, rounded exactly as a host computation without FMA
template <typename T>
__global__ void k_probs(const typename C2<T>::t* __restrict__ a, uint64_t n, double* __restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        auto x = a[i];
        double re = x.x, im = x.y;
        out[i] = __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
    }
}

int reduction_grid(rq_state* s) { return rq::num_sms(s->device) * 4; }

// finalize `nout` partial rows and copy them to host
int finish(rq_state* s, unsigned nblocks, unsigned stride, unsigned nout, double* host) {
    double* dout = s->partials + (size_t)nout * stride;
    k_finalize<<<nout, TPB, 0, s->stream>>>(s->partials, nblocks, stride, dout);
    RQ_CUDA(cudaGetLastError());
    RQ_TRY(rq::ensure_hbuf(s, nout));
    RQ_CUDA(cudaMemcpyAsync(s->hbuf, dout, nout * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    RQ_TRY(rq::sync_checked(s));
    for (unsigned k = 0; k < nout; ++k) host[k] = s->hbuf[k];
    return RQ_OK;
}

inline double re_ipow(uint32_t k) {
    switch (k & 3u) {
        case 0: return 1.0;
        case 2: return -1.0;
        default: return 0.0;
    }
}

}  // namespace

namespace rq {

int prob_bit(rq_state* s, uint32_t q, int want_one, double* out) {
    unsigned G = reduction_grid(s);
    uint64_t count = q < 64 ? s->n >> 1 : s->n;
    G = std::min<unsigned>(G, grid_for(count, TPB, num_sms(s->device), 4));
    RQ_TRY(ensure_partials(s, 2 * (size_t)G + 8));
    if (s->prec == RQ_F32)
        k_prob<float><<<G, TPB, 0, s->stream>>>((const float2*)s->amps, count, q, want_one, s->partials);
    else
        k_prob<double><<<G, TPB, 0, s->stream>>>((const double2*)s->amps, count, q, want_one, s->partials);
    RQ_CUDA(cudaGetLastError());
    return finish(s, G, G, 1, out);
}

int norm_sq(rq_state* s, double* out) { return prob_bit(s, 64, 0, out); }

int pauli_expect(rq_state* s, const PauliMask* terms, uint32_t nterms, double* out) {
    if (nterms == 0) return RQ_OK;
    unsigned G = reduction_grid(s);
    RQ_TRY(ensure_partials(s, (size_t)nterms * G + nterms + 8));
    std::vector<uint32_t> slot_of(nterms);
    uint32_t slot = 0;
    // single-qubit Z strings and identities: one pass for up to ZMAX of them
    std::vector<uint32_t> zs;
    if (s->nq >= 10)
        for (uint32_t k = 0; k < nterms; ++k)
            if (terms[k].xmask == 0 && __builtin_popcountll(terms[k].pmask) <= 1) zs.push_back(k);
    for (size_t c0 = 0; c0 < zs.size(); c0 += ZMAX) {
        ZChunk zc{};
        zc.k = (int)std::min<size_t>(ZMAX, zs.size() - c0);
        for (int k = 0; k < zc.k; ++k) {
            const uint64_t pm = terms[zs[c0 + k]].pmask;
            zc.q[k] = (uint8_t)(pm ? __builtin_ctzll(pm) : 64);
            slot_of[zs[c0 + k]] = slot + k;
        }
        const uint64_t nseg = s->n >> 10;     // segments of 1024 amplitudes, one warp each
        const unsigned Gz = std::min<unsigned>(G, grid_for(nseg * 32, TPB, num_sms(s->device), 4));
        if (s->prec == RQ_F32)
            k_zsingle<float><<<Gz, TPB, 0, s->stream>>>((const float2*)s->amps, nseg, zc, s->partials, slot, G);
        else
            k_zsingle<double><<<Gz, TPB, 0, s->stream>>>((const double2*)s->amps, nseg, zc, s->partials, slot, G);
        RQ_CUDA(cudaGetLastError());
        // blocks past Gz contribute nothing to these rows
        if (Gz < G)
            for (int k = 0; k < zc.k; ++k)
                RQ_CUDA(cudaMemsetAsync(s->partials + (size_t)(slot + k) * G + Gz, 0, (G - Gz) * sizeof(double),
                                        s->stream));
        slot += zc.k;
    }
    std::vector<char> done(nterms, 0);
    for (uint32_t k : zs) done[k] = 1;
    // the other strings: group by xmask (stable), chunks of KMAX
    std::map<uint64_t, std::vector<uint32_t>> groups;
    for (uint32_t k = 0; k < nterms; ++k)
        if (!done[k]) groups[terms[k].xmask].push_back(k);
    for (auto& kv : groups) {
        uint64_t x = kv.first;
        uint32_t h = x ? 63 - __builtin_clzll(x) : 0;
        uint64_t count = x ? s->n >> 1 : s->n;
        const auto& idx = kv.second;
        for (size_t c0 = 0; c0 < idx.size(); c0 += KMAX) {
            TermChunk tc{};
            tc.k = (int)std::min<size_t>(KMAX, idx.size() - c0);
            for (int k = 0; k < tc.k; ++k) {
                const PauliMask& t = terms[idx[c0 + k]];
                tc.pmask[k] = t.pmask;
                tc.odd[k] = x ? (__builtin_popcountll(x & t.pmask) & 1) : 0;
                slot_of[idx[c0 + k]] = slot + k;
            }
            if (s->prec == RQ_F32)
                k_pauli<float><<<G, TPB, 0, s->stream>>>((const float2*)s->amps, count, x, h, tc, s->partials, slot, G);
            else
                k_pauli<double><<<G, TPB, 0, s->stream>>>((const double2*)s->amps, count, x, h, tc, s->partials, slot, G);
            RQ_CUDA(cudaGetLastError());
            slot += tc.k;
        }
    }
    std::vector<double> sums(nterms);
    RQ_TRY(finish(s, G, G, nterms, sums.data()));
    for (uint32_t k = 0; k < nterms; ++k) {
        const PauliMask& t = terms[k];
        double acc = sums[slot_of[k]];
        if (t.xmask == 0) {
            out[k] = acc * re_ipow(t.ny);
        } else if (!(__builtin_popcountll(t.xmask & t.pmask) & 1)) {
            out[k] = 2.0 * acc * re_ipow(t.ny);
        } else {
            out[k] = 2.0 * acc * re_ipow(t.ny + 1);
        }
    }
    return RQ_OK;
}

int inner(rq_state* a, rq_state* b, double* re, double* im) {
    unsigned G = reduction_grid(a);
    RQ_TRY(ensure_partials(a, 2 * (size_t)G + 8));
    // b's pending work must be done before a's stream reads it
    RQ_CUDA(cudaStreamSynchronize(b->stream));
    if (a->prec == RQ_F32 && b->prec == RQ_F32)
        k_inner<float, float><<<G, TPB, 0, a->stream>>>((const float2*)a->amps, (const float2*)b->amps, a->n, a->partials, G);
    else if (a->prec == RQ_F32)
        k_inner<float, double><<<G, TPB, 0, a->stream>>>((const float2*)a->amps, (const double2*)b->amps, a->n, a->partials, G);
    else if (b->prec == RQ_F32)
        k_inner<double, float><<<G, TPB, 0, a->stream>>>((const double2*)a->amps, (const float2*)b->amps, a->n, a->partials, G);
    else
        k_inner<double, double><<<G, TPB, 0, a->stream>>>((const double2*)a->amps, (const double2*)b->amps, a->n, a->partials, G);
    RQ_CUDA(cudaGetLastError());
    double r[2];
    RQ_TRY(finish(a, G, G, 2, r));
    *re = r[0];
    *im = r[1];
    return RQ_OK;
}

int probabilities_dev(rq_state* s, double* dev_out) {
    unsigned g = grid_for(s->n, TPB, num_sms(s->device));
    if (s->prec == RQ_F32) k_probs<float><<<g, TPB, 0, s->stream>>>((const float2*)s->amps, s->n, dev_out);
    else k_probs<double><<<g, TPB, 0, s->stream>>>((const double2*)s->amps, s->n, dev_out);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

}  // namespace rq

// ---------------------------------------------------------------------------
// Allocation-free expectation values (rq_expectation_batch_noalloc).
//
// Some callers cannot allocate device memory at all (their budget is fixed, or
// another framework owns the allocator).  For them the partial sums of the
// Pauli-string reduction live in this one static device array instead of the
// per-state buffer.  It is fixed in size, exists once per GPU that loads the
// library, and is shared by every call: two calls in flight at once on the GPU
// would overwrite each other's partials, so callers must serialise them.
// Nothing in it has to start at zero: every slot a call reads back was
// written by that same call's first kernel.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_noalloc_scratch[RQ_NOALLOC_SCRATCH_DOUBLES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_addr[kMaxDevices] = {nullptr};
unsigned long long g_noalloc_ctx[kMaxDevices] = {0};   // context the address belongs to

// Unique id of the current CUDA context (cuCtxGetId, reached through the runtime's
// driver entry points so the library needs no libcuda link); 0 when unavailable.
unsigned long long current_context_id() {
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        return cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
                       q == cudaDriverEntryPointSuccess ? reinterpret_cast<GetCurrent>(f) : nullptr;
    }();
    static GetId get_id = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        return cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
                       q == cudaDriverEntryPointSuccess ? reinterpret_cast<GetId>(f) : nullptr;
    }();
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of g_noalloc_scratch on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// with that device current, once per device and context: the first call on a
// device (and the first call after its context was re-created, for example by
// cudaDeviceReset, which reloads the module and can move the array) looks it
// up; later calls reuse it.
int noalloc_scratch_address(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "device index out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    const unsigned long long ctx = current_context_id();
    if (!g_noalloc_addr[device] || ctx == 0 || ctx != g_noalloc_ctx[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return rq::cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_addr[device] = static_cast<double*>(p);
        g_noalloc_ctx[device] = ctx;
    }
    *out = g_noalloc_addr[device];
    return RQ_OK;
}

}  // namespace

extern "C" int rq_expectation_batch_noalloc(const void* device_amps, uint32_t num_qubits, int32_t precision,
                                            const rq_pauli_op* ops, const uint32_t* offsets, uint32_t nstrings,
                                            double* out, void* stream_handle) {
    if (!device_amps || (!out && nstrings) || (!offsets && nstrings))
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (precision != RQ_F32 && precision != RQ_F64)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "precision must be RQ_F32 or RQ_F64");
    uint32_t maxq = precision == RQ_F32 ? RQ_MAX_QUBITS_F32 : RQ_MAX_QUBITS_F64;
    if (num_qubits == 0 || num_qubits > maxq)
        return rq::fail(RQ_ERR_QUBIT_LIMIT_EXCEEDED, "num_qubits must be in 1.." + std::to_string(maxq));
    if (nstrings > RQ_NOALLOC_MAX_STRINGS)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "rq_expectation_batch_noalloc takes at most " +
                                                     std::to_string(RQ_NOALLOC_MAX_STRINGS) + " Pauli strings per call, got " +
                                                     std::to_string(nstrings));
    if (nstrings == 0) return RQ_OK;
    if (!ops && offsets[nstrings] > offsets[0]) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    // Pauli strings in mask form (same rules as rq_state_expectation_batch)
    std::vector<rq::PauliMask> terms(nstrings);
    for (uint32_t k = 0; k < nstrings; ++k) {
        if (offsets[k + 1] < offsets[k]) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "offsets must be non-decreasing");
        rq::PauliMask m{0, 0, 0};
        for (uint32_t j = offsets[k]; j < offsets[k + 1]; ++j) {
            uint32_t q = ops[j].qubit;
            int op = ops[j].op;
            if (op < RQ_PAULI_I || op > RQ_PAULI_Z)
                return rq::fail(RQ_ERR_INVALID_ARGUMENT, "invalid Pauli operator " + std::to_string(op));
            if (op == RQ_PAULI_I) continue;
            if (q >= num_qubits)
                return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "invalid qubit index " + std::to_string(q) + " for " +
                                                                std::to_string(num_qubits) + "-qubit system");
            uint64_t b = 1ull << q;
            if (op == RQ_PAULI_X || op == RQ_PAULI_Y) m.xmask ^= b;
            if (op == RQ_PAULI_Y || op == RQ_PAULI_Z) m.pmask ^= b;
            if (op == RQ_PAULI_Y) m.ny += 1;
        }
        m.ny &= 3u;
        terms[k] = m;
    }
    int device = 0;
    RQ_CUDA(cudaGetDevice(&device));
    double* scratch = nullptr;
    RQ_TRY(noalloc_scratch_address(device, &scratch));
    cudaStream_t st = static_cast<cudaStream_t>(stream_handle);
    const uint64_t n = 1ull << num_qubits;
    unsigned G = (unsigned)std::min<int>(rq::num_sms(device) * 4, (int)RQ_NOALLOC_MAX_BLOCKS);
    // partials occupy [0, nstrings*G); the finalised sums follow at nstrings*G
    std::map<uint64_t, std::vector<uint32_t>> groups;
    for (uint32_t k = 0; k < nstrings; ++k) groups[terms[k].xmask].push_back(k);
    std::vector<uint32_t> slot_of(nstrings);
    uint32_t slot = 0;
    for (auto& kv : groups) {
        uint64_t x = kv.first;
        uint32_t h = x ? 63 - __builtin_clzll(x) : 0;
        uint64_t count = x ? n >> 1 : n;
        const auto& idx = kv.second;
        for (size_t c0 = 0; c0 < idx.size(); c0 += KMAX) {
            TermChunk tc{};
            tc.k = (int)std::min<size_t>(KMAX, idx.size() - c0);
            for (int k = 0; k < tc.k; ++k) {
                const rq::PauliMask& t = terms[idx[c0 + k]];
                tc.pmask[k] = t.pmask;
                tc.odd[k] = x ? (__builtin_popcountll(x & t.pmask) & 1) : 0;
                slot_of[idx[c0 + k]] = slot + k;
            }
            if (precision == RQ_F32)
                k_pauli<float><<<G, TPB, 0, st>>>((const float2*)device_amps, count, x, h, tc, scratch, slot, G);
            else
                k_pauli<double><<<G, TPB, 0, st>>>((const double2*)device_amps, count, x, h, tc, scratch, slot, G);
            RQ_CUDA(cudaGetLastError());
            slot += tc.k;
        }
    }
    double* sums = scratch + (size_t)nstrings * G;
    k_finalize<<<nstrings, TPB, 0, st>>>(scratch, G, G, sums);
    RQ_CUDA(cudaGetLastError());
    std::vector<double> host(nstrings);
    RQ_CUDA(cudaMemcpyAsync(host.data(), sums, nstrings * sizeof(double), cudaMemcpyDeviceToHost, st));
    RQ_CUDA(cudaStreamSynchronize(st));
    for (uint32_t k = 0; k < nstrings; ++k) {
        const rq::PauliMask& t = terms[k];
        double acc = host[slot_of[k]];
        if (t.xmask == 0) out[k] = acc * re_ipow(t.ny);
        else if (!(__builtin_popcountll(t.xmask & t.pmask) & 1)) out[k] = 2.0 * acc * re_ipow(t.ny);
        else out[k] = 2.0 * acc * re_ipow(t.ny + 1);
    }
    return RQ_OK;
}
