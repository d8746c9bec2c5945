// rq_gates.cu -- one-kernel-per-gate path (the unfused execution mode).
//
// Each kernel is one pass over the amplitudes that the gate touches; these
// are the B200 counterparts of apply_single_qubit_gate (state.rs:214-229)
// and apply_two_qubit_gate (state.rs:238-276), with the 2q loop enumerating
// only the 2^(n-2) valid groups instead of skipping 3/4 of all bases, and
// with permutation (CNOT, SWAP) and diagonal (CZ, Rzz, Rz, ...) gates
// touching only the amplitudes they change.
#include "rq_internal.cuh"

namespace {

using rqd::C2;
using rqd::insert0;

template <typename T>
struct CM2 { T v[8]; };    // 2x2 complex, (re,im) row-major
template <typename T>
struct CM4 { T v[32]; };   // 4x4 complex
template <typename T>
struct CD4 { T v[8]; };    // 4 complex diagonal entries

template <typename V, typename T>
__device__ __forceinline__ V cmac2(T ar, T ai, V x, T br, T bi, V y) {
    // (a*x + b*y) with a=(ar,ai), b=(br,bi)
    V r;
    r.x = ar * x.x - ai * x.y + br * y.x - bi * y.y;
    r.y = ar * x.y + ai * x.x + br * y.y + bi * y.x;
    return r;
}

template <typename T>
__global__ void k_gate1q(typename C2<T>::t* __restrict__ a, uint64_t npairs, uint32_t q, CM2<T> m) {
    using V = typename C2<T>::t;
    const uint64_t step = 1ull << q;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npairs;
         p += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i0 = insert0(p, q), i1 = i0 | step;
        V x = a[i0], y = a[i1];
        a[i0] = cmac2<V, T>(m.v[0], m.v[1], x, m.v[2], m.v[3], y);
        a[i1] = cmac2<V, T>(m.v[4], m.v[5], x, m.v[6], m.v[7], y);
    }
}

// qubit 0, f32: the pair is one 16-byte vector
__global__ void k_gate1q_q0_f32(float4* __restrict__ a, uint64_t npairs, CM2<float> m) {
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npairs;
         p += (uint64_t)gridDim.x * blockDim.x) {
        float4 v = a[p];
        float2 x = make_float2(v.x, v.y), y = make_float2(v.z, v.w);
        float2 o0 = cmac2<float2, float>(m.v[0], m.v[1], x, m.v[2], m.v[3], y);
        float2 o1 = cmac2<float2, float>(m.v[4], m.v[5], x, m.v[6], m.v[7], y);
        a[p] = make_float4(o0.x, o0.y, o1.x, o1.y);
    }
}

// diag(d0, d1) on qubit q; when d0 == 1 only the bit=1 half is touched
template <typename T>
__global__ void k_diag1q(typename C2<T>::t* __restrict__ a, uint64_t count, uint32_t q, int half_only, CD4<T> d) {
    using V = typename C2<T>::t;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < count;
         p += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i = half_only ? (insert0(p, q) | (1ull << q)) : p;
        int b = (int)((i >> q) & 1);
        T dr = d.v[2 * b], di = d.v[2 * b + 1];
        V x = a[i];
        V r;
        r.x = dr * x.x - di * x.y;
        r.y = dr * x.y + di * x.x;
        a[i] = r;
    }
}

template <typename T>
__global__ void k_gate2q(typename C2<T>::t* __restrict__ a, uint64_t ngroups, uint32_t q1, uint32_t q2, CM4<T> m) {
    using V = typename C2<T>::t;
    const uint32_t lo = q1 < q2 ? q1 : q2, hi = q1 < q2 ? q2 : q1;
    const uint64_t b1 = 1ull << q1, b2 = 1ull << q2;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t base = insert0(insert0(g, lo), hi);
        uint64_t idx[4] = {base, base | b2, base | b1, base | b1 | b2};
        V v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = a[idx[k]];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            V acc = cmac2<V, T>(m.v[8 * r + 0], m.v[8 * r + 1], v[0], m.v[8 * r + 2], m.v[8 * r + 3], v[1]);
            V acc2 = cmac2<V, T>(m.v[8 * r + 4], m.v[8 * r + 5], v[2], m.v[8 * r + 6], m.v[8 * r + 7], v[3]);
            acc.x += acc2.x;
            acc.y += acc2.y;
            a[idx[r]] = acc;
        }
    }
}

// diagonal 4x4 over all amplitudes: a_i *= d[bit(q1)*2 + bit(q2)]
template <typename T>
__global__ void k_diag2q(typename C2<T>::t* __restrict__ a, uint64_t n, uint32_t q1, uint32_t q2, CD4<T> d) {
    using V = typename C2<T>::t;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        int k = (int)(((i >> q1) & 1) * 2 + ((i >> q2) & 1));
        T dr = d.v[2 * k], di = d.v[2 * k + 1];
        V x = a[i];
        V r;
        r.x = dr * x.x - di * x.y;
        r.y = dr * x.y + di * x.x;
        a[i] = r;
    }
}

// CNOT(c,t): swap the target pair inside the control=1 half
template <typename T>
__global__ void k_cnot(typename C2<T>::t* __restrict__ a, uint64_t ngroups, uint32_t c, uint32_t t) {
    using V = typename C2<T>::t;
    const uint32_t lo = c < t ? c : t, hi = c < t ? t : c;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i = insert0(insert0(g, lo), hi) | (1ull << c);
        uint64_t j = i | (1ull << t);
        V x = a[i], y = a[j];
        a[i] = y;
        a[j] = x;
    }
}

template <typename T>
__global__ void k_swap(typename C2<T>::t* __restrict__ a, uint64_t ngroups, uint32_t q1, uint32_t q2) {
    using V = typename C2<T>::t;
    const uint32_t lo = q1 < q2 ? q1 : q2, hi = q1 < q2 ? q2 : q1;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t base = insert0(insert0(g, lo), hi);
        uint64_t i = base | (1ull << q2), j = base | (1ull << q1);
        V x = a[i], y = a[j];
        a[i] = y;
        a[j] = x;
    }
}

template <typename T>
__global__ void k_cz(typename C2<T>::t* __restrict__ a, uint64_t ngroups, uint32_t q1, uint32_t q2) {
    using V = typename C2<T>::t;
    const uint32_t lo = q1 < q2 ? q1 : q2, hi = q1 < q2 ? q2 : q1;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i = insert0(insert0(g, lo), hi) | (1ull << q1) | (1ull << q2);
        V x = a[i];
        x.x = -x.x;
        x.y = -x.y;
        a[i] = x;
    }
}

template <typename T>
__global__ void k_scale(typename C2<T>::t* __restrict__ a, uint64_t n, T f) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        auto x = a[i];
        x.x *= f;
        x.y *= f;
        a[i] = x;
    }
}

// measurement collapse (state.rs:306-317): keep the observed branch scaled
// by nf, zero the other one
template <typename T>
__global__ void k_collapse(typename C2<T>::t* __restrict__ a, uint64_t n, uint32_t q, int keep_one, T nf) {
    using V = typename C2<T>::t;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        int one = (int)((i >> q) & 1);
        V x = a[i];
        if (one == keep_one) {
            x.x *= nf;
            x.y *= nf;
        } else {
            x.x = 0;
            x.y = 0;
        }
        a[i] = x;
    }
}

template <typename T>
__global__ void k_from_f64(typename C2<T>::t* __restrict__ a, const double2* __restrict__ src, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        double2 v = src[i];
        typename C2<T>::t o;
        o.x = (T)v.x;
        o.y = (T)v.y;
        a[i] = o;
    }
}

template <typename T>
__global__ void k_to_f64(const typename C2<T>::t* __restrict__ a, double2* __restrict__ dst, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        auto v = a[i];
        dst[i] = make_double2((double)v.x, (double)v.y);
    }
}

// host amplitude edits of run_grover (grover.rs:128-153) as device passes
template <typename T>
__global__ void k_negate_except(typename C2<T>::t* __restrict__ a, uint64_t n, uint64_t keep) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        if (i == keep) continue;
        auto x = a[i];
        x.x = -x.x;
        x.y = -x.y;
        a[i] = x;
    }
}

// distinct indices (the host folds repeats), so no two threads touch one amplitude
template <typename T>
__global__ void k_negate_list(typename C2<T>::t* __restrict__ a, const uint64_t* __restrict__ idx, uint64_t count) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = idx[k];
        auto x = a[i];
        x.x = -x.x;
        x.y = -x.y;
        a[i] = x;
    }
}

// one half of the amplitudes (bit q == v), in the order of the other bits, to / from a
// contiguous buffer: the exchange step of a state split over ranks by its top qubits
template <typename T>
__global__ void k_half_copy(typename C2<T>::t* __restrict__ a, typename C2<T>::t* __restrict__ buf, uint64_t half,
                            uint32_t q, uint32_t v, int unpack) {
    const uint64_t lo = (1ull << q) - 1;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < half;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t idx = ((i & ~lo) << 1) | ((uint64_t)v << q) | (i & lo);
        if (unpack) a[idx] = buf[i];
        else buf[i] = a[idx];
    }
}

template <typename T>
__global__ void k_basis(typename C2<T>::t* __restrict__ a, uint64_t n, uint64_t index) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        typename C2<T>::t v;
        v.x = i == index ? (T)1 : (T)0;
        v.y = 0;
        a[i] = v;
    }
}

template <typename T>
CM2<T> cm2(const double* m8) {
    CM2<T> r;
    for (int k = 0; k < 8; ++k) r.v[k] = (T)m8[k];
    return r;
}

constexpr int TPB = 256;

}  // namespace

namespace rq {

#define RQ_LAUNCH(kernel, work, ...)                                                    \
    do {                                                                               \
        unsigned g_ = grid_for((work), TPB, num_sms(s->device));                       \
        kernel<<<g_, TPB, 0, s->stream>>>(__VA_ARGS__);                                \
        RQ_CUDA(cudaGetLastError());                                                   \
    } while (0)

// |index>: one write pass, no host transfer (so it is stream-ordered and capturable)
int init_basis(rq_state* s, uint64_t index) {
    if (s->prec == RQ_F32) RQ_LAUNCH(k_basis<float>, s->n, (float2*)s->amps, s->n, index);
    else RQ_LAUNCH(k_basis<double>, s->n, (double2*)s->amps, s->n, index);
    return RQ_OK;
}


int gate1q(rq_state* s, uint32_t q, const double* m8) {
    uint64_t np = s->n >> 1;
    if (s->prec == RQ_F32) {
        if (q == 0) RQ_LAUNCH(k_gate1q_q0_f32, np, (float4*)s->amps, np, cm2<float>(m8));
        else RQ_LAUNCH(k_gate1q<float>, np, (float2*)s->amps, np, q, cm2<float>(m8));
    } else {
        RQ_LAUNCH(k_gate1q<double>, np, (double2*)s->amps, np, q, cm2<double>(m8));
    }
    return RQ_OK;
}

int gate1q_diag(rq_state* s, uint32_t q, const double* d4) {
    int half = (d4[0] == 1.0 && d4[1] == 0.0) ? 1 : 0;
    uint64_t cnt = half ? s->n >> 1 : s->n;
    if (s->prec == RQ_F32) {
        CD4<float> d; for (int k = 0; k < 4; ++k) d.v[k] = (float)d4[k];
        RQ_LAUNCH(k_diag1q<float>, cnt, (float2*)s->amps, cnt, q, half, d);
    } else {
        CD4<double> d; for (int k = 0; k < 4; ++k) d.v[k] = d4[k];
        RQ_LAUNCH(k_diag1q<double>, cnt, (double2*)s->amps, cnt, q, half, d);
    }
    return RQ_OK;
}

int gate2q(rq_state* s, uint32_t q1, uint32_t q2, const double* m32) {
    uint64_t ng = s->n >> 2;
    if (s->prec == RQ_F32) {
        CM4<float> m; for (int k = 0; k < 32; ++k) m.v[k] = (float)m32[k];
        RQ_LAUNCH(k_gate2q<float>, ng, (float2*)s->amps, ng, q1, q2, m);
    } else {
        CM4<double> m; for (int k = 0; k < 32; ++k) m.v[k] = m32[k];
        RQ_LAUNCH(k_gate2q<double>, ng, (double2*)s->amps, ng, q1, q2, m);
    }
    return RQ_OK;
}

int gate2q_diag(rq_state* s, uint32_t q1, uint32_t q2, const double* d8) {
    if (s->prec == RQ_F32) {
        CD4<float> d; for (int k = 0; k < 8; ++k) d.v[k] = (float)d8[k];
        RQ_LAUNCH(k_diag2q<float>, s->n, (float2*)s->amps, s->n, q1, q2, d);
    } else {
        CD4<double> d; for (int k = 0; k < 8; ++k) d.v[k] = d8[k];
        RQ_LAUNCH(k_diag2q<double>, s->n, (double2*)s->amps, s->n, q1, q2, d);
    }
    return RQ_OK;
}

int gate_cnot(rq_state* s, uint32_t c, uint32_t t) {
    uint64_t ng = s->n >> 2;
    if (s->prec == RQ_F32) RQ_LAUNCH(k_cnot<float>, ng, (float2*)s->amps, ng, c, t);
    else RQ_LAUNCH(k_cnot<double>, ng, (double2*)s->amps, ng, c, t);
    return RQ_OK;
}

int gate_swap(rq_state* s, uint32_t q1, uint32_t q2) {
    uint64_t ng = s->n >> 2;
    if (s->prec == RQ_F32) RQ_LAUNCH(k_swap<float>, ng, (float2*)s->amps, ng, q1, q2);
    else RQ_LAUNCH(k_swap<double>, ng, (double2*)s->amps, ng, q1, q2);
    return RQ_OK;
}

int gate_cz(rq_state* s, uint32_t q1, uint32_t q2) {
    uint64_t ng = s->n >> 2;
    if (s->prec == RQ_F32) RQ_LAUNCH(k_cz<float>, ng, (float2*)s->amps, ng, q1, q2);
    else RQ_LAUNCH(k_cz<double>, ng, (double2*)s->amps, ng, q1, q2);
    return RQ_OK;
}

int half_copy(rq_state* s, uint32_t q, uint32_t v, void* buf, int unpack) {
    const uint64_t half = s->n >> 1;
    if (s->prec == RQ_F32) RQ_LAUNCH(k_half_copy<float>, half, (float2*)s->amps, (float2*)buf, half, q, v, unpack);
    else RQ_LAUNCH(k_half_copy<double>, half, (double2*)s->amps, (double2*)buf, half, q, v, unpack);
    return RQ_OK;
}

int negate_except(rq_state* s, uint64_t keep) {
    if (s->prec == RQ_F32) RQ_LAUNCH(k_negate_except<float>, s->n, (float2*)s->amps, s->n, keep);
    else RQ_LAUNCH(k_negate_except<double>, s->n, (double2*)s->amps, s->n, keep);
    return RQ_OK;
}

int negate_list(rq_state* s, const uint64_t* dev_idx, uint64_t count) {
    if (count == 0) return RQ_OK;
    if (s->prec == RQ_F32) RQ_LAUNCH(k_negate_list<float>, count, (float2*)s->amps, dev_idx, count);
    else RQ_LAUNCH(k_negate_list<double>, count, (double2*)s->amps, dev_idx, count);
    return RQ_OK;
}

int scale_all(rq_state* s, double f) {
    if (s->prec == RQ_F32) RQ_LAUNCH(k_scale<float>, s->n, (float2*)s->amps, s->n, (float)f);
    else RQ_LAUNCH(k_scale<double>, s->n, (double2*)s->amps, s->n, f);
    return RQ_OK;
}

int collapse(rq_state* s, uint32_t q, int keep_one, double nf) {
    if (s->prec == RQ_F32) RQ_LAUNCH(k_collapse<float>, s->n, (float2*)s->amps, s->n, q, keep_one, (float)nf);
    else RQ_LAUNCH(k_collapse<double>, s->n, (double2*)s->amps, s->n, q, keep_one, nf);
    return RQ_OK;
}

int upload_f64(rq_state* s, const double* src) {
    if (s->prec == RQ_F32) RQ_LAUNCH(k_from_f64<float>, s->n, (float2*)s->amps, (const double2*)src, s->n);
    else RQ_CUDA(cudaMemcpyAsync(s->amps, src, s->bytes(), cudaMemcpyDeviceToDevice, s->stream));
    return RQ_OK;
}

int download_f64(rq_state* s, double* dst) {
    if (s->prec == RQ_F32) RQ_LAUNCH(k_to_f64<float>, s->n, (const float2*)s->amps, (double2*)dst, s->n);
    else RQ_CUDA(cudaMemcpyAsync(dst, s->amps, s->bytes(), cudaMemcpyDeviceToDevice, s->stream));
    return RQ_OK;
}

}  // namespace rq
