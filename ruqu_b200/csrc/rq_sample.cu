// rq_sample.cu -- shot sampling without collapse.
//
// Simulator::run_shots (simulator.rs:107-147) re-simulates the circuit once
// per shot and measures qubit after qubit (state.rs:288-335): outcome 1 iff
// u >= P(q = 0 | earlier outcomes).  Here the circuit runs once; the
// probabilities are folded into a prefix tree over the measured qubits (in
// measurement order) and every shot walks the tree with the same uniforms
// (draw k of key base_seed + shot), so each shot reproduces the reference's
// sequential conditional sampling.  FP64 throughout, sums without FMA so a
// host fold of the same probability vector gives identical bits.
#include "rq_internal.cuh"

#include <vector>

namespace {

using rqd::C2;

constexpr int TPB = 256;
constexpr int MAXQ = 64;

struct Perm {
    uint8_t order[MAXQ];   // permuted bit position -> qubit
    uint8_t pos[MAXQ];     // qubit -> permuted bit position
    uint32_t n;
    int identity;
};

struct Plan {
    uint8_t qubits[MAXQ];  // measurement order (may repeat)
    uint32_t m;
};

__device__ __forceinline__ uint64_t unpermute(uint64_t j, const Perm& P) {
    if (P.identity) return j;
    uint64_t i = 0;
    for (uint32_t b = 0; b < P.n; ++b) i |= ((j >> b) & 1ull) << P.order[b];
    return i;
}

template <typename T>
__device__ __forceinline__ double prob_at(const typename C2<T>::t* a, uint64_t i) {
    auto x = a[i];
    double re = x.x, im = x.y;
    return __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
}

// level n-1 of the tree straight from the amplitudes
template <typename T>
__global__ void k_leaf_fold(const typename C2<T>::t* __restrict__ a, Perm P, double* __restrict__ lvl) {
    const uint64_t half = 1ull << (P.n - 1);
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < half;
         j += (uint64_t)gridDim.x * blockDim.x) {
        double p0 = prob_at<T>(a, unpermute(j, P));
        double p1 = prob_at<T>(a, unpermute(j + half, P));
        lvl[j] = __dadd_rn(p0, p1);
    }
}

// level k from level k+1 (both 2^k / 2^(k+1) long)
__global__ void k_fold(const double* __restrict__ up, double* __restrict__ dn, uint64_t len) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < len;
         j += (uint64_t)gridDim.x * blockDim.x)
        dn[j] = __dadd_rn(up[j], up[j + len]);
}

// all levels from `top` down to 0 in one block (top level has <= 2^12 entries)
__global__ void k_fold_tail(double* __restrict__ tree, int top) {
    for (int k = top - 1; k >= 0; --k) {
        const double* up = tree + ((1ull << (k + 1)) - 1);
        double* dn = tree + ((1ull << k) - 1);
        uint64_t len = 1ull << k;
        for (uint64_t j = threadIdx.x; j < len; j += blockDim.x) dn[j] = __dadd_rn(up[j], up[j + len]);
        __syncthreads();
    }
}

template <typename T>
__global__ void k_sample(const typename C2<T>::t* __restrict__ a, const double* __restrict__ tree, Perm P,
                         Plan plan, uint64_t base_seed, uint64_t shots, uint64_t* __restrict__ out) {
    for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < shots;
         s += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t key = base_seed + s;
        uint64_t prefix = 0, bits = 0, done = 0, val = 0;
        for (uint32_t k = 0; k < plan.m; ++k) {
            uint32_t q = plan.qubits[k];
            int r;
            if ((done >> q) & 1ull) {
                r = (int)((val >> q) & 1ull);
            } else {
                uint32_t lev = P.pos[q];
                double m0, m1;
                if (lev + 1 == P.n) {
                    m0 = prob_at<T>(a, unpermute(prefix, P));
                    m1 = prob_at<T>(a, unpermute(prefix | (1ull << lev), P));
                } else {
                    const double* L = tree + ((1ull << (lev + 1)) - 1);
                    m0 = L[prefix];
                    m1 = L[prefix | (1ull << lev)];
                }
                double p0 = m0 / __dadd_rn(m0, m1);
                double u = rqd::uniform(key, 0, k);
                r = u >= p0 ? 1 : 0;
                prefix |= (uint64_t)r << lev;
                done |= 1ull << q;
                val |= (uint64_t)r << q;
            }
            if (r) bits |= 1ull << q;
            else bits &= ~(1ull << q);
        }
        out[s] = bits;
    }
}

// out[i] = entry index[i] of tree level `level` (level n: |a|^2 at that permuted index)
template <typename T>
__global__ void k_tree_lookup(const typename C2<T>::t* __restrict__ a, const double* __restrict__ tree, Perm P,
                              uint32_t level, const uint64_t* __restrict__ index, uint64_t count,
                              double* __restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t j = index[i];
        out[i] = level == P.n ? prob_at<T>(a, unpermute(j, P)) : tree[((1ull << level) - 1) + j];
    }
}

}  // namespace

namespace rq {

namespace {

// The permutation of a tree over `qubits` (first appearance order; the other qubits after them).
Perm make_perm(uint32_t n, const uint32_t* qubits, uint32_t nqm) {
    Perm P{};
    P.n = n;
    std::vector<int> pos(n, -1);
    uint32_t next = 0;
    for (uint32_t k = 0; k < nqm; ++k)
        if (pos[qubits[k]] < 0) { pos[qubits[k]] = (int)next; P.order[next++] = (uint8_t)qubits[k]; }
    for (uint32_t q = 0; q < n; ++q)
        if (pos[q] < 0) { pos[q] = (int)next; P.order[next++] = (uint8_t)q; }
    P.identity = 1;
    for (uint32_t q = 0; q < n; ++q) {
        P.pos[q] = (uint8_t)pos[q];
        if (pos[q] != (int)q) P.identity = 0;
    }
    return P;
}

Perm stored_perm(const rq_state* s) {
    Perm P{};
    P.n = s->nq;
    P.identity = 1;
    for (uint32_t b = 0; b < s->nq; ++b) {
        P.order[b] = s->tree_order[b];
        P.pos[s->tree_order[b]] = (uint8_t)b;
        if (s->tree_order[b] != b) P.identity = 0;
    }
    return P;
}

// tree levels 0..n-1 at offsets 2^k - 1 (level n is the probability vector itself)
int build_tree(rq_state* s, const Perm& P) {
    const uint32_t n = s->nq;
    s->tree_ready = false;
    RQ_TRY(ensure_tree(s, (size_t)1 << n));
    int sms = num_sms(s->device);
    double* top = s->tree + ((1ull << (n - 1)) - 1);
    uint64_t half = 1ull << (n - 1);
    unsigned g = grid_for(half, TPB, sms);
    if (s->prec == RQ_F32) k_leaf_fold<float><<<g, TPB, 0, s->stream>>>((const float2*)s->amps, P, top);
    else k_leaf_fold<double><<<g, TPB, 0, s->stream>>>((const double2*)s->amps, P, top);
    RQ_CUDA(cudaGetLastError());
    int k = (int)n - 2;
    for (; k >= 0 && (1ull << (k + 1)) > 4096; --k) {
        double* up = s->tree + ((1ull << (k + 1)) - 1);
        double* dn = s->tree + ((1ull << k) - 1);
        uint64_t len = 1ull << k;
        k_fold<<<grid_for(len, TPB, sms), TPB, 0, s->stream>>>(up, dn, len);
        RQ_CUDA(cudaGetLastError());
    }
    if (k >= 0) {
        k_fold_tail<<<1, 1024, 0, s->stream>>>(s->tree, k + 1);
        RQ_CUDA(cudaGetLastError());
    }
    for (uint32_t b = 0; b < n; ++b) s->tree_order[b] = P.order[b];
    s->tree_ready = true;
    return RQ_OK;
}

}  // namespace

int sample(rq_state* s, const uint32_t* qubits, uint32_t nqm, uint64_t base_seed, uint64_t shots,
           uint64_t* host_out) {
    if (shots == 0) return RQ_OK;
    const uint32_t n = s->nq;
    if (n > 63 || nqm > MAXQ) return fail(RQ_ERR_INVALID_ARGUMENT, "sampling supports at most 63 qubits and 64 measurements");
    const Perm P = make_perm(n, qubits, nqm);
    Plan plan{};
    plan.m = nqm;
    for (uint32_t k = 0; k < nqm; ++k) plan.qubits[k] = (uint8_t)qubits[k];
    RQ_TRY(build_tree(s, P));
    const int sms = num_sms(s->device);
    uint64_t* dout = nullptr;
    RQ_CUDA(cudaMallocAsync((void**)&dout, shots * sizeof(uint64_t), s->stream));
    unsigned gs = grid_for(shots, 128, sms);
    if (s->prec == RQ_F32)
        k_sample<float><<<gs, 128, 0, s->stream>>>((const float2*)s->amps, s->tree, P, plan, base_seed, shots, dout);
    else
        k_sample<double><<<gs, 128, 0, s->stream>>>((const double2*)s->amps, s->tree, P, plan, base_seed, shots, dout);
    cudaError_t le = cudaGetLastError();
    cudaError_t ce = cudaMemcpyAsync(host_out, dout, shots * sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream);
    cudaFreeAsync(dout, s->stream);
    RQ_CUDA(le);
    RQ_CUDA(ce);
    return rq::sync_checked(s);
}

int tree_build(rq_state* s, const uint32_t* qubits, uint32_t nqm) {
    if (s->nq > 63) return fail(RQ_ERR_INVALID_ARGUMENT, "prefix trees support at most 63 qubits");
    RQ_TRY(build_tree(s, make_perm(s->nq, qubits, nqm)));
    return rq::sync_checked(s);
}

int tree_lookup(rq_state* s, uint32_t level, const uint64_t* index, uint64_t count, double* host_out) {
    if (!s->tree_ready) return fail(RQ_ERR_INVALID_ARGUMENT, "no prefix tree: build one first");
    if (level > s->nq) return fail(RQ_ERR_INVALID_ARGUMENT, "tree level above the qubit count");
    const uint64_t lim = 1ull << level;
    for (uint64_t i = 0; i < count; ++i)
        if (index[i] >= lim) return fail(RQ_ERR_INVALID_ARGUMENT, "tree index out of range for its level");
    if (count == 0) return RQ_OK;
    const Perm P = stored_perm(s);
    uint64_t* didx = nullptr;
    double* dout = nullptr;
    RQ_CUDA(cudaMallocAsync((void**)&didx, count * sizeof(uint64_t), s->stream));
    cudaError_t e = cudaMallocAsync((void**)&dout, count * sizeof(double), s->stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(didx, s->stream);
        return cuda_fail(e, "tree lookup buffers");
    }
    e = cudaMemcpyAsync(didx, index, count * sizeof(uint64_t), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) {
        const unsigned g = grid_for(count, TPB, num_sms(s->device));
        if (s->prec == RQ_F32)
            k_tree_lookup<float><<<g, TPB, 0, s->stream>>>((const float2*)s->amps, s->tree, P, level, didx, count, dout);
        else
            k_tree_lookup<double><<<g, TPB, 0, s->stream>>>((const double2*)s->amps, s->tree, P, level, didx, count, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_out, dout, count * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    cudaFreeAsync(didx, s->stream);
    cudaFreeAsync(dout, s->stream);
    RQ_CUDA(e);
    return rq::sync_checked(s);
}

}  // namespace rq
