// rq_internal.cuh -- shared internals of libruqu_cuda.so (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include "../../include/ruqu_cuda.h"

// Opaque state handle of the C ABI: one device buffer of 2^n interleaved
// complex amplitudes (float2 or double2), one stream, the measurement stream
// position, and lazily grown device scratch.
struct rq_state {
    uint32_t nq = 0;
    int32_t prec = RQ_F64;
    uint64_t n = 0;               // 2^nq
    void* amps = nullptr;         // float2* or double2*
    cudaStream_t stream = nullptr;
    int device = 0;
    uint64_t seed = 0;
    uint64_t draws = 0;           // next draw index of measurement stream 0
    double* partials = nullptr;   // reduction partials
    size_t partials_cap = 0;      // in doubles
    double* tree = nullptr;       // sampling prefix tree (levels 0..n-1)
    size_t tree_cap = 0;          // in doubles
    uint8_t tree_order[64] = {};  // the tree's bit k -> qubit (measured qubits first)
    bool tree_ready = false;      // tree holds the levels of tree_order (rq_state_tree_build / sample)
    double* hbuf = nullptr;       // pinned host staging for small results
    size_t hbuf_cap = 0;          // in doubles
    int32_t exec_mode = RQ_EXEC_AUTO;
    size_t elem_bytes() const { return prec == RQ_F32 ? 8 : 16; }
    size_t bytes() const { return (size_t)n * elem_bytes(); }
};

namespace rq {

// ---- errors -------------------------------------------------------------
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
#define RQ_CUDA(call)                                                   \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return ::rq::cuda_fail(e_, #call);       \
    } while (0)
#define RQ_TRY(expr)                                                    \
    do {                                                                \
        int rc_ = (expr);                                               \
        if (rc_ != RQ_OK) return rc_;                                   \
    } while (0)

// ---- device facts --------------------------------------------------------
int num_sms(int device);

// Grid for a grid-stride loop over `work` items: at most 8 resident
// 256-thread blocks per SM, never more blocks than needed.
inline unsigned grid_for(uint64_t work, int threads, int sms, int per_sm = 8) {
    uint64_t need = (work + threads - 1) / threads;
    uint64_t cap = (uint64_t)sms * per_sm;
    if (need < 1) need = 1;
    return (unsigned)(need < cap ? need : cap);
}

// ---- scratch ----------------------------------------------------------------
int ensure_partials(rq_state* s, size_t ndoubles);
int ensure_hbuf(rq_state* s, size_t ndoubles);
int ensure_tree(rq_state* s, size_t ndoubles);

// ---- kernels' host launchers (rq_gates.cu) --------------------------------
int init_basis(rq_state* s, uint64_t index);
int gate1q(rq_state* s, uint32_t q, const double* m8);        // generic 2x2
int gate1q_diag(rq_state* s, uint32_t q, const double* d4);   // diag(d0, d1)
int gate2q(rq_state* s, uint32_t q1, uint32_t q2, const double* m32);
int gate2q_diag(rq_state* s, uint32_t q1, uint32_t q2, const double* d8);
int gate_cnot(rq_state* s, uint32_t c, uint32_t t);
int gate_swap(rq_state* s, uint32_t q1, uint32_t q2);
int gate_cz(rq_state* s, uint32_t q1, uint32_t q2);
int scale_all(rq_state* s, double f);
int negate_except(rq_state* s, uint64_t keep);
int half_copy(rq_state* s, uint32_t q, uint32_t v, void* device_buf, int unpack);
int negate_list(rq_state* s, const uint64_t* dev_idx, uint64_t count);   // distinct indices < 2^n
int collapse(rq_state* s, uint32_t q, int keep_one, double nf);
int upload_f64(rq_state* s, const double* dev_interleaved);   // device f64 -> state
int download_f64(rq_state* s, double* dev_interleaved);       // state -> device f64

// ---- reductions (rq_reduce.cu) ---------------------------------------------
// Pauli string in mask form: xmask = XOR of X/Y qubits, pmask = XOR of
// Y/Z qubits, ny = number of Y factors (mod 4).  This reproduces the
// reference's per-factor loop (state.rs:366-395) exactly, including repeated
// qubits, because that loop reads every factor's bit from the original index.
struct PauliMask {
    uint64_t xmask;
    uint64_t pmask;
    uint32_t ny;
};
int norm_sq(rq_state* s, double* out);
int prob_bit(rq_state* s, uint32_t q, int want_one, double* out);
int pauli_expect(rq_state* s, const PauliMask* terms, uint32_t nterms, double* out);
int inner(rq_state* a, rq_state* b, double* re, double* im);
int probabilities_dev(rq_state* s, double* dev_out);

// ---- sampling (rq_sample.cu) -------------------------------------------------
int sample(rq_state* s, const uint32_t* qubits, uint32_t nq, uint64_t base_seed,
           uint64_t shots, uint64_t* host_out);
int tree_build(rq_state* s, const uint32_t* qubits, uint32_t nq);
int tree_lookup(rq_state* s, uint32_t level, const uint64_t* index, uint64_t count, double* host_out);

// ---- fused sweeps and prepared plans (rq_sweep.cu) ---------------------------
// tc_passes > 0: fuse each phase's slot-local gate runs into dense 32x32 unitaries
// on the tensor cores (3 = 3xTF32, 1 = one TF32 pass); complex f32, m in {12, 13}
// m > 0 overrides the number of local qubits of a sweep (the tile shape)
int apply_sweeps(rq_state* s, const rq_gate* gates, uint64_t n, int tc_passes = 0, uint32_t m = 0);
int plan_build(const rq_state* s, const rq_gate* gates, uint64_t n, int32_t mode, rq_plan** out, int tc_passes = 0,
               uint32_t tc_min_ops = 2, uint32_t m = 0);
// RQ_EXEC_AUTO's measured choice of execution (CUDA-core sweep, or 3xTF32 tensor-core sweep
// with 13 or 12 local qubits): tensor-core passes (0 or 3) and tile shape (m, 0 = default),
// cached per (device, qubits, gate structure)
int autotune_tc(const rq_state* s, const rq_gate* gates, uint64_t n, int* passes, uint32_t* m);
// the tensor-core arithmetic a mode asks for: 0 none, 3 = 3xTF32, 1 = one TF32 pass,
// TC_F16 = three FP16 passes (RQ_EXEC_SWEEP_TC16)
constexpr int TC_F16 = 16;
inline int tc_passes_of(int32_t mode) {
    return mode == RQ_EXEC_SWEEP_TC ? 3 : mode == RQ_EXEC_SWEEP_TC_FAST ? 1 : mode == RQ_EXEC_SWEEP_TC16 ? TC_F16 : 0;
}
int plan_launch(rq_state* s, const rq_plan* p);
// the same gate kinds and qubits as the plan was built for (barriers ignored)
bool plan_same_shape(const rq_plan* p, const rq_gate* gates, uint64_t n);
// new gate values for a plan of the same structure (RQ_ERR_CIRCUIT, plan unchanged, otherwise)
int plan_rebind(rq_state* s, rq_plan* p, const rq_gate* gates, uint64_t n);
void plan_free(rq_plan* p);
rq_plan_stats plan_stats(const rq_plan* p);
bool plan_fits(const rq_plan* p, const rq_state* s);
int apply_one_gate(rq_state* s, const rq_gate& g);   // per-gate kernels (rq_capi.cu)

// ---- tensor-core GEMM (rq_mlp.cu) -------------------------------------------
// read-and-clear of the GEMM kernels' expired-wait flag on the current device
int mma_timeout_flag(int* out);
// polls before an mbarrier wait counts as expired (0: the default), current device
int mma_set_wait_polls(uint32_t polls);
// the tensor-core sweeps' equivalents (rq_sweep.cu)
int tc_timeout_flag(int* out);
int tc_set_wait_polls(uint32_t polls);
// synchronise the state's stream, then report (and clear) an expired tensor-core wait as
// RQ_ERR_TIMEOUT: the read-back paths call this, so a sweep that gave up is never read as
// if it had finished
int sync_checked(rq_state* s);

}  // namespace rq

// ---- device helpers -----------------------------------------------------------
namespace rqd {

template <typename T> struct C2;
template <> struct C2<float> { using t = float2; };
template <> struct C2<double> { using t = double2; };

// insert a zero bit at position b of x
__host__ __device__ __forceinline__ uint64_t insert0(uint64_t x, uint32_t b) {
    uint64_t lo = x & ((1ull << b) - 1);
    return ((x >> b) << (b + 1)) | lo;
}

// Philox4x32-10 (Salmon et al., SC'11), same stream as rq_uniform().
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k0 += W0; k1 += W1; }
        uint64_t p0 = (uint64_t)M0 * c[0];
        uint64_t p1 = (uint64_t)M1 * c[2];
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    }
}

__host__ __device__ __forceinline__ double uniform(uint64_t seed, uint32_t stream, uint64_t index) {
    uint64_t blk = index >> 1;
    uint32_t c[4] = {(uint32_t)blk, (uint32_t)(blk >> 32), stream, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint32_t hi = (index & 1) ? c[2] : c[0];
    uint32_t lo = (index & 1) ? c[3] : c[1];
    uint64_t w = ((uint64_t)hi << 32) | lo;
    return (double)(w >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace rqd
