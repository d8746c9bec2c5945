// rq_capi.cu -- the extern "C" boundary (include/ruqu_cuda.h).
//
// Host-side validation mirrors QuantumState::apply_gate (state.rs:158-204)
// and the constructors (state.rs:31-96); gate matrices are built on the host
// in f64 exactly as Gate::matrix_1q / matrix_2q do (gate.rs:72-198) and are
// narrowed to f32 for f32 states like convert_matrix_1q/2q
// (mixed_precision.rs:556-591).  Kernels live in rq_gates.cu, rq_reduce.cu,
// rq_sample.cu and rq_sweep.cu; nothing here computes on amplitudes.
#include "rq_internal.cuh"

#include <algorithm>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

namespace {

thread_local std::string g_last_error;

const double kFrac1Sqrt2 = 0.70710678118654752440;

bool is_2q(int k) { return k == RQ_GATE_CNOT || k == RQ_GATE_CZ || k == RQ_GATE_SWAP || k == RQ_GATE_RZZ; }

// Gate::matrix_1q (gate.rs:72-146) as 8 doubles, (re,im) row-major
bool matrix_1q(const rq_gate& g, double m[8]) {
    auto set = [&](double a, double b, double c, double d, double e, double f, double h, double i) {
        m[0] = a; m[1] = b; m[2] = c; m[3] = d; m[4] = e; m[5] = f; m[6] = h; m[7] = i;
    };
    const double s = kFrac1Sqrt2;
    switch (g.kind) {
        case RQ_GATE_H: set(s, 0, s, 0, s, 0, -s, -0.0); return true;
        case RQ_GATE_X: set(0, 0, 1, 0, 1, 0, 0, 0); return true;
        case RQ_GATE_Y: set(0, 0, -0.0, -1, 0, 1, 0, 0); return true;
        case RQ_GATE_Z: set(1, 0, 0, 0, 0, 0, -1, -0.0); return true;
        case RQ_GATE_S: set(1, 0, 0, 0, 0, 0, 0, 1); return true;
        case RQ_GATE_SDG: set(1, 0, 0, 0, 0, 0, -0.0, -1); return true;
        case RQ_GATE_T: set(1, 0, 0, 0, 0, 0, s, s); return true;
        case RQ_GATE_TDG: set(1, 0, 0, 0, 0, 0, s, -s); return true;
        case RQ_GATE_RX: {
            double h = g.angle / 2.0, c = std::cos(h), sn = -std::sin(h);
            set(c, 0, 0, sn, 0, sn, c, 0); return true;
        }
        case RQ_GATE_RY: {
            double h = g.angle / 2.0, c = std::cos(h), sn = std::sin(h);
            set(c, 0, -sn, 0, sn, 0, c, 0); return true;
        }
        case RQ_GATE_RZ: {
            double h = g.angle / 2.0;
            set(std::cos(-h), std::sin(-h), 0, 0, 0, 0, std::cos(h), std::sin(h)); return true;
        }
        case RQ_GATE_PHASE: set(1, 0, 0, 0, 0, 0, std::cos(g.angle), std::sin(g.angle)); return true;
        case RQ_GATE_UNITARY1Q: std::memcpy(m, g.m, sizeof(double) * 8); return true;
        default: return false;
    }
}

bool is_diag_1q(int k) {
    return k == RQ_GATE_Z || k == RQ_GATE_S || k == RQ_GATE_SDG || k == RQ_GATE_T || k == RQ_GATE_TDG ||
           k == RQ_GATE_RZ || k == RQ_GATE_PHASE;
}

int validate_gate(const rq_state* s, const rq_gate& g) {
    if (g.kind < RQ_GATE_H || g.kind > RQ_GATE_UNITARY1Q)
        return rq::fail(RQ_ERR_CIRCUIT, "circuit error: unsupported gate kind " + std::to_string(g.kind));
    if (g.kind == RQ_GATE_BARRIER) return RQ_OK;
    uint32_t qs[2] = {g.q0, g.q1};
    int nq = is_2q(g.kind) ? 2 : 1;
    for (int k = 0; k < nq; ++k)
        if (qs[k] >= s->nq)
            return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "invalid qubit index " + std::to_string(qs[k]) + " for " +
                                                            std::to_string(s->nq) + "-qubit system");
    if (nq == 2 && g.q0 == g.q1)
        return rq::fail(RQ_ERR_CIRCUIT, "circuit error: two-qubit gate requires distinct qubits, got " +
                                            std::to_string(g.q0) + " and " + std::to_string(g.q1));
    return RQ_OK;
}

int device_of_current() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}

int set_device(const rq_state* s) {
    RQ_CUDA(cudaSetDevice(s->device));
    return RQ_OK;
}

int check_create(uint32_t nq, int32_t prec) {
    if (prec != RQ_F32 && prec != RQ_F64) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "precision must be RQ_F32 or RQ_F64");
    uint32_t maxq = prec == RQ_F32 ? RQ_MAX_QUBITS_F32 : RQ_MAX_QUBITS_F64;
    if (nq == 0) return rq::fail(RQ_ERR_CIRCUIT, "circuit error: cannot create quantum state with 0 qubits");
    if (nq > maxq)
        return rq::fail(RQ_ERR_QUBIT_LIMIT_EXCEEDED, "qubit limit exceeded: requested " + std::to_string(nq) +
                                                         ", maximum " + std::to_string(maxq));
    return RQ_OK;
}

int alloc_state(uint32_t nq, int32_t prec, uint64_t seed, rq_state** out) {
    rq_state* s = new rq_state();
    s->nq = nq;
    s->prec = prec;
    s->n = 1ull << nq;
    s->seed = seed;
    s->device = device_of_current();
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        return rq::cuda_fail(e, "cudaStreamCreateWithFlags");
    }
    e = cudaMalloc(&s->amps, s->bytes());
    if (e != cudaSuccess) {
        cudaGetLastError();
        size_t need = s->bytes();
        cudaStreamDestroy(s->stream);
        delete s;
        return rq::fail(RQ_ERR_MEMORY_ALLOCATION, "memory allocation failed: need " + std::to_string(need) + " bytes");
    }
    *out = s;
    return RQ_OK;
}

uint64_t entropy_seed() {
    std::random_device rd;
    return ((uint64_t)rd() << 32) ^ rd();
}

int to_masks(const rq_state* s, const rq_pauli_op* ops, uint32_t nops, rq::PauliMask* m) {
    m->xmask = 0;
    m->pmask = 0;
    m->ny = 0;
    for (uint32_t k = 0; k < nops; ++k) {
        uint32_t q = ops[k].qubit;
        int op = ops[k].op;
        if (op < RQ_PAULI_I || op > RQ_PAULI_Z)
            return rq::fail(RQ_ERR_INVALID_ARGUMENT, "invalid Pauli operator " + std::to_string(op));
        if (op == RQ_PAULI_I) continue;
        if (q >= s->nq)
            return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "invalid qubit index " + std::to_string(q) + " for " +
                                                            std::to_string(s->nq) + "-qubit system");
        uint64_t b = 1ull << q;
        if (op == RQ_PAULI_X || op == RQ_PAULI_Y) m->xmask ^= b;
        if (op == RQ_PAULI_Y || op == RQ_PAULI_Z) m->pmask ^= b;
        if (op == RQ_PAULI_Y) m->ny += 1;
    }
    m->ny &= 3u;
    return RQ_OK;
}

int do_measure(rq_state* s, uint32_t q, rq_measurement* out) {
    double p0 = 0.0;
    RQ_TRY(rq::prob_bit(s, q, 0, &p0));
    double u = rqd::uniform(s->seed, 0, s->draws++);
    int result = u >= p0 ? 1 : 0;
    double prob = result ? 1.0 - p0 : p0;
    double nf = prob > 0.0 ? 1.0 / std::sqrt(prob) : 0.0;
    RQ_TRY(rq::collapse(s, q, result, nf));
    if (out) {
        out->qubit = q;
        out->result = result;
        out->probability = prob;
    }
    return RQ_OK;
}

int do_reset(rq_state* s, uint32_t q) {
    rq_measurement m;
    RQ_TRY(do_measure(s, q, &m));
    if (m.result) {
        double x[8] = {0, 0, 1, 0, 1, 0, 0, 0};
        RQ_TRY(rq::gate1q(s, q, x));
    }
    return RQ_OK;
}

}  // namespace

// one unitary gate through the per-gate kernels
int rq::apply_one_gate(rq_state* s, const rq_gate& g) {
    switch (g.kind) {
        case RQ_GATE_CNOT: return rq::gate_cnot(s, g.q0, g.q1);
        case RQ_GATE_CZ: return rq::gate_cz(s, g.q0, g.q1);
        case RQ_GATE_SWAP: return rq::gate_swap(s, g.q0, g.q1);
        case RQ_GATE_RZZ: {
            double h = g.angle / 2.0;
            double en_r = std::cos(-h), en_i = std::sin(-h), ep_r = std::cos(h), ep_i = std::sin(h);
            double d[8] = {en_r, en_i, ep_r, ep_i, ep_r, ep_i, en_r, en_i};
            return rq::gate2q_diag(s, g.q0, g.q1, d);
        }
        default: break;
    }
    double m[8];
    if (!matrix_1q(g, m)) return rq::fail(RQ_ERR_CIRCUIT, "circuit error: unsupported gate");
    if (is_diag_1q(g.kind)) {
        double d[4] = {m[0], m[1], m[6], m[7]};
        return rq::gate1q_diag(s, g.q0, d);
    }
    return rq::gate1q(s, g.q0, m);
}

namespace {

bool is_unitary(int k) { return k != RQ_GATE_MEASURE && k != RQ_GATE_RESET && k != RQ_GATE_BARRIER; }

}  // namespace

// ===========================================================================
// internal helpers shared by the translation units
// ===========================================================================
namespace rq {

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
    return RQ_ERR_CUDA;
}

int num_sms(int device) {
    static std::mutex mu;
    static int cache[64] = {0};
    if (device < 0 || device >= 64) return 148;
    std::lock_guard<std::mutex> lk(mu);
    if (cache[device] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0) v = 148;
        cache[device] = v;
    }
    return cache[device];
}

int ensure_partials(rq_state* s, size_t nd) {
    if (s->partials_cap >= nd) return RQ_OK;
    if (s->partials) {
        RQ_CUDA(cudaStreamSynchronize(s->stream));
        cudaFree(s->partials);
        s->partials = nullptr;
        s->partials_cap = 0;
    }
    size_t cap = nd < 4096 ? 4096 : nd;
    RQ_CUDA(cudaMalloc(&s->partials, cap * sizeof(double)));
    s->partials_cap = cap;
    return RQ_OK;
}

int ensure_hbuf(rq_state* s, size_t nd) {
    if (s->hbuf_cap >= nd) return RQ_OK;
    if (s->hbuf) {
        RQ_CUDA(cudaStreamSynchronize(s->stream));
        cudaFreeHost(s->hbuf);
        s->hbuf = nullptr;
        s->hbuf_cap = 0;
    }
    size_t cap = nd < 1024 ? 1024 : nd;
    RQ_CUDA(cudaMallocHost(&s->hbuf, cap * sizeof(double)));
    s->hbuf_cap = cap;
    return RQ_OK;
}

int ensure_tree(rq_state* s, size_t nd) {
    if (s->tree_cap >= nd) return RQ_OK;
    if (s->tree) {
        RQ_CUDA(cudaStreamSynchronize(s->stream));
        cudaFree(s->tree);
        s->tree = nullptr;
        s->tree_cap = 0;
    }
    cudaError_t e = cudaMalloc(&s->tree, nd * sizeof(double));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(RQ_ERR_MEMORY_ALLOCATION, "memory allocation failed: need " + std::to_string(nd * sizeof(double)) +
                                                  " bytes of sampling scratch");
    }
    s->tree_cap = nd;
    return RQ_OK;
}

}  // namespace rq

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* rq_last_error_message(void) { return g_last_error.c_str(); }

int32_t rq_version(void) { return 100; }

double rq_uniform(uint64_t seed, uint32_t stream, uint64_t index) { return rqd::uniform(seed, stream, index); }

int rq_state_create(uint32_t num_qubits, int32_t precision, uint64_t seed, int32_t seeded, rq_state** out) {
    if (!out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null output pointer");
    RQ_TRY(check_create(num_qubits, precision));
    rq_state* s = nullptr;
    RQ_TRY(alloc_state(num_qubits, precision, seeded ? seed : entropy_seed(), &s));
    int rc = rq::init_basis(s, 0);
    if (rc == RQ_OK) {
        cudaError_t e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) rc = rq::cuda_fail(e, "cudaStreamSynchronize");
    }
    if (rc != RQ_OK) {
        rq_state_destroy(s);
        return rc;
    }
    *out = s;
    return RQ_OK;
}

int rq_state_from_amplitudes(const double* interleaved, uint64_t len, uint32_t num_qubits, int32_t precision,
                             uint64_t seed, rq_state** out) {
    if (!out || (!interleaved && len)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (precision != RQ_F32 && precision != RQ_F64)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "precision must be RQ_F32 or RQ_F64");
    uint32_t maxq = precision == RQ_F32 ? RQ_MAX_QUBITS_F32 : RQ_MAX_QUBITS_F64;
    if (num_qubits > maxq)
        return rq::fail(RQ_ERR_QUBIT_LIMIT_EXCEEDED, "qubit limit exceeded: requested " + std::to_string(num_qubits) +
                                                         ", maximum " + std::to_string(maxq));
    if (num_qubits == 0 || len != (1ull << num_qubits))
        return rq::fail(RQ_ERR_INVALID_STATE_VECTOR, "invalid state vector: length " + std::to_string(len) +
                                                         " does not match 2^" + std::to_string(num_qubits));
    rq_state* s = nullptr;
    RQ_TRY(alloc_state(num_qubits, precision, seed, &s));
    int rc = rq_state_upload(s, interleaved);
    if (rc != RQ_OK) {
        rq_state_destroy(s);
        return rc;
    }
    *out = s;
    return RQ_OK;
}

int rq_device_set(int32_t device) {
    RQ_CUDA(cudaSetDevice(device));
    return RQ_OK;
}

int rq_device_count(int32_t* out) {
    if (!out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    int n = 0;
    RQ_CUDA(cudaGetDeviceCount(&n));
    *out = n;
    return RQ_OK;
}

int rq_plan_create(const rq_state* s, const rq_gate* gates, uint64_t n, int32_t mode, rq_plan** out) {
    if (!s || !out || (!gates && n)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (mode < RQ_EXEC_AUTO || mode > RQ_EXEC_SWEEP_TC16)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "bad execution mode");
    for (uint64_t k = 0; k < n; ++k) {
        RQ_TRY(validate_gate(s, gates[k]));
        if (gates[k].kind == RQ_GATE_MEASURE || gates[k].kind == RQ_GATE_RESET)
            return rq::fail(RQ_ERR_CIRCUIT, "circuit error: a plan holds unitary gates only");
    }
    RQ_TRY(set_device(s));
    int use_sweep = (mode != RQ_EXEC_PER_GATE && (mode != RQ_EXEC_AUTO || s->nq >= 12)) && s->nq >= 7;
    int passes = rq::tc_passes_of(mode);
    uint32_t m = 0;
    if (mode == RQ_EXEC_AUTO && use_sweep) RQ_TRY(rq::autotune_tc(s, gates, n, &passes, &m));
    return rq::plan_build(s, gates, n, use_sweep ? RQ_EXEC_SWEEP : RQ_EXEC_PER_GATE, out, passes, 2, m);
}

int rq_plan_create_tiled(const rq_state* s, const rq_gate* gates, uint64_t n, int32_t mode, uint32_t local_qubits,
                         rq_plan** out) {
    if (local_qubits == 0) return rq_plan_create(s, gates, n, mode, out);
    if (!s || !out || (!gates && n)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    const uint32_t hi = mode == RQ_EXEC_SWEEP_TC16 ? 14u : 13u;
    if ((mode != RQ_EXEC_SWEEP_TC && mode != RQ_EXEC_SWEEP_TC_FAST && mode != RQ_EXEC_SWEEP_TC16) ||
        s->prec != RQ_F32 || local_qubits < 12 || local_qubits > hi || s->nq < local_qubits)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "tile sizes: 12-13 local qubits for the tensor-core sweeps, 12-14 for "
                                                 "RQ_EXEC_SWEEP_TC16, complex f32 states of at least that many qubits");
    for (uint64_t k = 0; k < n; ++k) {
        RQ_TRY(validate_gate(s, gates[k]));
        if (gates[k].kind == RQ_GATE_MEASURE || gates[k].kind == RQ_GATE_RESET)
            return rq::fail(RQ_ERR_CIRCUIT, "circuit error: a plan holds unitary gates only");
    }
    RQ_TRY(set_device(s));
    return rq::plan_build(s, gates, n, RQ_EXEC_SWEEP, out, rq::tc_passes_of(mode), 2, local_qubits);
}

int rq_state_apply_kraus(rq_state* s, uint32_t q, const double* kraus, uint32_t nk, int32_t* chosen,
                         double* probability) {
    if (!s || (!kraus && nk)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (nk == 0 || nk > RQ_KRAUS_MAX)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "a channel has 1.." + std::to_string(RQ_KRAUS_MAX) + " Kraus operators");
    if (q >= s->nq)
        return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "invalid qubit index " + std::to_string(q) + " for " +
                                                        std::to_string(s->nq) + "-qubit system");
    RQ_TRY(set_device(s));
    // the qubit's reduced density matrix rho_ij = sum a_i conj(a_j) over the pairs of amplitudes
    // that differ in bit q, from <I>, <Z_q>, <X_q>, <Y_q> (FP64 reductions on the device)
    const uint64_t b = 1ull << q;
    const rq::PauliMask t[4] = {{0, 0, 0}, {0, b, 0}, {b, 0, 0}, {b, b, 1}};
    double ev[4];
    RQ_TRY(rq::pauli_expect(s, t, 4, ev));
    const double r00 = 0.5 * (ev[0] + ev[1]), r11 = 0.5 * (ev[0] - ev[1]);
    const double r01r = 0.5 * ev[2], r01i = -0.5 * ev[3];   // rho_10 = conj(rho_01)
    // p_k = tr(K_k rho K_k^dagger)
    std::vector<double> pk(nk);
    double total = 0.0;
    for (uint32_t k = 0; k < nk; ++k) {
        const double* K = kraus + 8 * (size_t)k;   // row-major 2x2, (re, im) pairs
        double acc = 0.0;
        for (int i = 0; i < 2; ++i) {
            const double ar = K[4 * i], ai = K[4 * i + 1], br = K[4 * i + 2], bi = K[4 * i + 3];
            // (K rho K^dagger)_ii = |a|^2 r00 + |b|^2 r11 + 2 Re(a rho01 conj(b))
            const double cr = ar * r01r - ai * r01i, ci = ar * r01i + ai * r01r;   // a rho01
            acc += (ar * ar + ai * ai) * r00 + (br * br + bi * bi) * r11 + 2.0 * (cr * br + ci * bi);
        }
        pk[k] = acc > 0.0 ? acc : 0.0;
        total += pk[k];
    }
    if (!(total > 0.0)) return rq::fail(RQ_ERR_INVALID_STATE_VECTOR, "the channel annihilates the state");
    const double u = rqd::uniform(s->seed, 0, s->draws++);
    uint32_t pick = nk - 1;
    double cum = 0.0;
    for (uint32_t k = 0; k < nk; ++k) {
        cum += pk[k] / total;
        if (u < cum && pk[k] > 0.0) {
            pick = k;
            break;
        }
    }
    while (pk[pick] == 0.0 && pick > 0) --pick;
    const double f = 1.0 / std::sqrt(pk[pick] / total);   // the state keeps its norm
    double m8[8];
    for (int j = 0; j < 8; ++j) m8[j] = kraus[8 * (size_t)pick + j] * f;
    RQ_TRY(rq::gate1q(s, q, m8));
    if (chosen) *chosen = (int32_t)pick;
    if (probability) *probability = pk[pick] / total;
    return RQ_OK;
}

int rq_plan_update(rq_state* s, rq_plan* p, const rq_gate* gates, uint64_t n) {
    if (!s || !p || (!gates && n)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (!rq::plan_fits(p, s))
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "plan was built for another qubit count, precision or device");
    for (uint64_t k = 0; k < n; ++k) {
        RQ_TRY(validate_gate(s, gates[k]));
        if (gates[k].kind == RQ_GATE_MEASURE || gates[k].kind == RQ_GATE_RESET)
            return rq::fail(RQ_ERR_CIRCUIT, "circuit error: a plan holds unitary gates only");
    }
    RQ_TRY(set_device(s));
    return rq::plan_rebind(s, p, gates, n);
}

int rq_plan_execute(rq_state* s, const rq_plan* p) {
    if (!s || !p) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (!rq::plan_fits(p, s))
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "plan was built for another qubit count, precision or device");
    RQ_TRY(set_device(s));
    return rq::plan_launch(s, p);
}

int rq_plan_get_stats(const rq_plan* p, rq_plan_stats* out) {
    if (!p || !out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    *out = rq::plan_stats(p);
    return RQ_OK;
}

int rq_plan_destroy(rq_plan* p) {
    rq::plan_free(p);
    return RQ_OK;
}

int rq_state_destroy(rq_state* s) {
    if (!s) return RQ_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->amps) cudaFree(s->amps);
    if (s->partials) cudaFree(s->partials);
    if (s->tree) cudaFree(s->tree);
    if (s->hbuf) cudaFreeHost(s->hbuf);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return RQ_OK;
}

int rq_state_reset(rq_state* s) {
    if (!s) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null state");
    RQ_TRY(set_device(s));
    s->draws = 0;
    return rq::init_basis(s, 0);   // stream-ordered; later calls on s see the reset state
}

int rq_state_num_qubits(const rq_state* s, uint32_t* out) {
    if (!s || !out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    *out = s->nq;
    return RQ_OK;
}

int rq_state_precision(const rq_state* s, int32_t* out) {
    if (!s || !out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    *out = s->prec;
    return RQ_OK;
}

int rq_state_device_ptr(const rq_state* s, void** out_ptr, void** out_stream) {
    if (!s) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null state");
    if (out_ptr) *out_ptr = s->amps;
    if (out_stream) *out_stream = (void*)s->stream;
    return RQ_OK;
}

int rq_state_synchronize(rq_state* s) {
    if (!s) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null state");
    RQ_TRY(set_device(s));
    return rq::sync_checked(s);
}

int rq_debug_set_wait_limit(uint32_t polls) {
    RQ_TRY(rq::tc_set_wait_polls(polls));
    return rq::mma_set_wait_polls(polls);
}

}  // extern "C"

namespace {

// The gate loop of run_with_config (simulator.rs:67-78) over a validated list:
// measurements and resets in order, every maximal run of unitary gates through the
// sweep path (or per-gate kernels).  With mdraw, the k-th measurement / reset of the
// list takes draw index mdraw[k] of the state's stream (noise draws interleave).
int run_gate_list(rq_state* s, const rq_gate* gates, uint64_t n, int32_t mode, rq_measurement* out, uint64_t cap,
                  uint64_t* nout, const uint64_t* mdraw) {
    // states below 7 qubits are smaller than one sweep tile: per-gate kernels
    int use_sweep = (mode != RQ_EXEC_PER_GATE && (mode != RQ_EXEC_AUTO || s->nq >= 12)) && s->nq >= 7;
    uint64_t nm = 0, nmr = 0;
    uint64_t k = 0;
    while (k < n) {
        const rq_gate& g = gates[k];
        if (g.kind == RQ_GATE_BARRIER) { ++k; continue; }
        if (g.kind == RQ_GATE_MEASURE || g.kind == RQ_GATE_RESET) {
            if (mdraw) s->draws = mdraw[nmr];
            ++nmr;
            rq_measurement m;
            if (g.kind == RQ_GATE_MEASURE) {
                RQ_TRY(do_measure(s, g.q0, &m));
                if (out && nm < cap) out[nm] = m;
                ++nm;
            } else {
                RQ_TRY(do_reset(s, g.q0));
            }
            ++k;
            continue;
        }
        // maximal run of unitary gates (barriers inside a run are no-ops)
        uint64_t e = k;
        while (e < n && (is_unitary(gates[e].kind) || gates[e].kind == RQ_GATE_BARRIER)) ++e;
        if (use_sweep) {
            std::vector<rq_gate> run;
            run.reserve(e - k);
            for (uint64_t j = k; j < e; ++j)
                if (gates[j].kind != RQ_GATE_BARRIER) run.push_back(gates[j]);
            int passes = rq::tc_passes_of(mode);
            uint32_t m = 0;
            if (mode == RQ_EXEC_AUTO) RQ_TRY(rq::autotune_tc(s, run.data(), run.size(), &passes, &m));
            RQ_TRY(rq::apply_sweeps(s, run.data(), run.size(), passes, m));
        } else {
            for (uint64_t j = k; j < e; ++j)
                if (gates[j].kind != RQ_GATE_BARRIER) RQ_TRY(rq::apply_one_gate(s, gates[j]));
        }
        k = e;
    }
    if (nout) *nout = nm;
    return RQ_OK;
}

rq_gate pauli_gate(int kind, uint32_t q) {
    rq_gate p{};
    p.kind = kind;
    p.q0 = q;
    return p;
}

}  // namespace

extern "C" {

int rq_state_apply_mode(rq_state* s, const rq_gate* gates, uint64_t n, int32_t mode, rq_measurement* out,
                        uint64_t cap, uint64_t* nout) {
    if (!s || (!gates && n)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (mode < RQ_EXEC_AUTO || mode > RQ_EXEC_SWEEP_TC16)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "bad execution mode");
    RQ_TRY(set_device(s));
    for (uint64_t k = 0; k < n; ++k) RQ_TRY(validate_gate(s, gates[k]));
    return run_gate_list(s, gates, n, mode, out, cap, nout, nullptr);
}

int rq_state_apply_noisy(rq_state* s, const rq_gate* gates, uint64_t n, const rq_noise_model* noise,
                         rq_measurement* out, uint64_t cap, uint64_t* nout) {
    if (!s || (!gates && n) || !noise) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_TRY(set_device(s));
    for (uint64_t k = 0; k < n; ++k) RQ_TRY(validate_gate(s, gates[k]));
    // The noise decisions depend on the stream only, not on the state: walk the list once
    // on the host, drawing in apply_noise's order (simulator.rs:177-221) -- per qubit of
    // each gate: depolarising r (and the Pauli choice when r < rate), bit-flip r, phase-flip
    // r -- with each measurement / reset keeping its own draw in between, and insert the
    // chosen Paulis after their gate.  The expanded list then runs on the device.
    const double dep = noise->depolarizing_rate, bf = noise->bit_flip_rate, pf = noise->phase_flip_rate;
    std::vector<rq_gate> ex;
    ex.reserve(n + n / 4);
    std::vector<uint64_t> mdraw;
    uint64_t d = s->draws;
    for (uint64_t k = 0; k < n; ++k) {
        const rq_gate& g = gates[k];
        if (g.kind == RQ_GATE_BARRIER) continue;   // Gate::qubits() is empty: no noise
        ex.push_back(g);
        if (g.kind == RQ_GATE_MEASURE || g.kind == RQ_GATE_RESET) mdraw.push_back(d++);
        const uint32_t qs[2] = {g.q0, g.q1};
        const int nq = is_2q(g.kind) ? 2 : 1;
        for (int j = 0; j < nq; ++j) {
            const uint32_t q = qs[j];
            if (dep > 0.0) {
                if (rqd::uniform(s->seed, 0, d++) < dep) {
                    const double c = rqd::uniform(s->seed, 0, d++);
                    ex.push_back(pauli_gate(c < 1.0 / 3.0 ? RQ_GATE_X : (c < 2.0 / 3.0 ? RQ_GATE_Y : RQ_GATE_Z), q));
                }
            }
            if (bf > 0.0 && rqd::uniform(s->seed, 0, d++) < bf) ex.push_back(pauli_gate(RQ_GATE_X, q));
            if (pf > 0.0 && rqd::uniform(s->seed, 0, d++) < pf) ex.push_back(pauli_gate(RQ_GATE_Z, q));
        }
    }
    const int rc = run_gate_list(s, ex.data(), ex.size(), s->exec_mode, out, cap, nout, mdraw.data());
    if (rc == RQ_OK) s->draws = d;
    return rc;
}

int rq_state_apply(rq_state* s, const rq_gate* gates, uint64_t n, rq_measurement* out, uint64_t cap,
                   uint64_t* nout) {
    return rq_state_apply_mode(s, gates, n, s ? s->exec_mode : RQ_EXEC_AUTO, out, cap, nout);
}

int rq_state_apply_1q_matrix(rq_state* s, uint32_t qubit, const double* m) {
    if (!s || !m) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (qubit >= s->nq)
        return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "invalid qubit index " + std::to_string(qubit) + " for " +
                                                        std::to_string(s->nq) + "-qubit system");
    RQ_TRY(set_device(s));
    return rq::gate1q(s, qubit, m);
}

int rq_state_apply_2q_matrix(rq_state* s, uint32_t q1, uint32_t q2, const double* m) {
    if (!s || !m) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    rq_gate g{};
    g.kind = RQ_GATE_CNOT;
    g.q0 = q1;
    g.q1 = q2;
    RQ_TRY(validate_gate(s, g));
    RQ_TRY(set_device(s));
    return rq::gate2q(s, q1, q2, m);
}

int rq_state_measure(rq_state* s, uint32_t qubit, rq_measurement* out) {
    if (!s || !out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (qubit >= s->nq)
        return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "invalid qubit index " + std::to_string(qubit) + " for " +
                                                        std::to_string(s->nq) + "-qubit system");
    RQ_TRY(set_device(s));
    return do_measure(s, qubit, out);
}

int rq_state_measure_all(rq_state* s, rq_measurement* out) {
    if (!s || !out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_TRY(set_device(s));
    for (uint32_t q = 0; q < s->nq; ++q) RQ_TRY(do_measure(s, q, &out[q]));
    return RQ_OK;
}

int rq_state_reset_qubit(rq_state* s, uint32_t qubit) {
    if (!s) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null state");
    if (qubit >= s->nq)
        return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "invalid qubit index " + std::to_string(qubit) + " for " +
                                                        std::to_string(s->nq) + "-qubit system");
    RQ_TRY(set_device(s));
    return do_reset(s, qubit);
}

int rq_state_sample(rq_state* s, const uint32_t* qubits, uint32_t nqubits, uint64_t base_seed, uint64_t shots,
                    uint64_t* out_bits) {
    if (!s || (!out_bits && shots) || (!qubits && nqubits)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    for (uint32_t k = 0; k < nqubits; ++k)
        if (qubits[k] >= s->nq)
            return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "invalid qubit index " + std::to_string(qubits[k]) + " for " +
                                                            std::to_string(s->nq) + "-qubit system");
    RQ_TRY(set_device(s));
    return rq::sample(s, qubits, nqubits, base_seed, shots, out_bits);
}

int rq_state_tree_build(rq_state* s, const uint32_t* qubits, uint32_t nqubits) {
    if (!s || (!qubits && nqubits)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (nqubits > 64) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "a prefix tree orders at most 64 qubits");
    for (uint32_t k = 0; k < nqubits; ++k)
        if (qubits[k] >= s->nq)
            return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "invalid qubit index " + std::to_string(qubits[k]) + " for " +
                                                            std::to_string(s->nq) + "-qubit system");
    RQ_TRY(set_device(s));
    return rq::tree_build(s, qubits, nqubits);
}

int rq_state_tree_lookup(rq_state* s, uint32_t level, const uint64_t* index, uint64_t count, double* out) {
    if (!s || ((!index || !out) && count)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_TRY(set_device(s));
    return rq::tree_lookup(s, level, index, count, out);
}

int rq_state_probabilities(rq_state* s, double* out) {
    if (!s || !out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_TRY(set_device(s));
    double* d = nullptr;
    RQ_CUDA(cudaMallocAsync((void**)&d, s->n * sizeof(double), s->stream));
    int rc = rq::probabilities_dev(s, d);
    cudaError_t e = cudaSuccess;
    if (rc == RQ_OK) e = cudaMemcpyAsync(out, d, s->n * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    cudaFreeAsync(d, s->stream);
    RQ_TRY(rc);
    RQ_CUDA(e);
    RQ_CUDA(cudaStreamSynchronize(s->stream));
    return RQ_OK;
}

int rq_state_probability_of_qubit(rq_state* s, uint32_t qubit, double* out) {
    if (!s || !out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (qubit >= s->nq)
        return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "invalid qubit index " + std::to_string(qubit) + " for " +
                                                        std::to_string(s->nq) + "-qubit system");
    RQ_TRY(set_device(s));
    return rq::prob_bit(s, qubit, 1, out);
}

int rq_state_expectation_value(rq_state* s, const rq_pauli_op* ops, uint32_t nops, double* out) {
    if (!s || !out || (!ops && nops)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    rq::PauliMask m;
    RQ_TRY(to_masks(s, ops, nops, &m));
    RQ_TRY(set_device(s));
    return rq::pauli_expect(s, &m, 1, out);
}

int rq_state_expectation_batch(rq_state* s, const rq_pauli_op* ops, const uint32_t* offsets, uint32_t nstrings,
                               double* out) {
    if (!s || (!out && nstrings) || (!offsets && nstrings)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (nstrings && !ops && offsets[nstrings] > offsets[0]) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    std::vector<rq::PauliMask> masks(nstrings);
    for (uint32_t k = 0; k < nstrings; ++k) {
        if (offsets[k + 1] < offsets[k]) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "offsets must be non-decreasing");
        RQ_TRY(to_masks(s, ops + offsets[k], offsets[k + 1] - offsets[k], &masks[k]));
    }
    RQ_TRY(set_device(s));
    return rq::pauli_expect(s, masks.data(), nstrings, out);
}

int rq_state_expectation_hamiltonian(rq_state* s, const double* coeffs, const rq_pauli_op* ops,
                                     const uint32_t* offsets, uint32_t nterms, double* out) {
    if (!out || (!coeffs && nterms)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    std::vector<double> ev(nterms);
    RQ_TRY(rq_state_expectation_batch(s, ops, offsets, nterms, ev.data()));
    double acc = 0.0;
    for (uint32_t k = 0; k < nterms; ++k) acc += coeffs[k] * ev[k];
    *out = acc;
    return RQ_OK;
}

int rq_state_norm_sq(rq_state* s, double* out) {
    if (!s || !out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_TRY(set_device(s));
    return rq::norm_sq(s, out);
}

int rq_state_normalize(rq_state* s) {
    double ns = 0.0;
    RQ_TRY(rq_state_norm_sq(s, &ns));
    if (ns > 0.0) RQ_TRY(rq::scale_all(s, 1.0 / std::sqrt(ns)));
    return RQ_OK;
}

int rq_state_negate_amplitudes(rq_state* s, const uint64_t* indices, uint64_t count) {
    if (!s || (!indices && count)) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    std::vector<uint64_t> v(indices, indices + count);
    for (uint64_t i : v)
        if (i >= s->n)
            return rq::fail(RQ_ERR_INVALID_ARGUMENT, "amplitude index " + std::to_string(i) + " out of range for " +
                                                         std::to_string(s->nq) + " qubits");
    // an index listed k times is negated k times: keep those with k odd, once each
    std::sort(v.begin(), v.end());
    std::vector<uint64_t> odd;
    for (size_t a = 0; a < v.size();) {
        size_t b = a;
        while (b < v.size() && v[b] == v[a]) ++b;
        if ((b - a) & 1) odd.push_back(v[a]);
        a = b;
    }
    if (odd.empty()) return RQ_OK;
    RQ_TRY(set_device(s));
    RQ_TRY(rq::ensure_partials(s, odd.size()));
    uint64_t* d_idx = reinterpret_cast<uint64_t*>(s->partials);
    RQ_CUDA(cudaMemcpyAsync(d_idx, odd.data(), odd.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, s->stream));
    RQ_TRY(rq::negate_list(s, d_idx, odd.size()));
    // the host list goes out of scope on return: finish the copy first
    RQ_CUDA(cudaStreamSynchronize(s->stream));
    return RQ_OK;
}

int rq_state_half_copy(rq_state* s, uint32_t qubit, uint32_t value, void* device_buf, int32_t direction) {
    if (!s || !device_buf) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (qubit >= s->nq)
        return rq::fail(RQ_ERR_INVALID_QUBIT_INDEX, "invalid qubit index " + std::to_string(qubit) + " for " +
                                                        std::to_string(s->nq) + "-qubit system");
    if (value > 1) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "value must be 0 or 1");
    if (direction != RQ_HALF_PACK && direction != RQ_HALF_UNPACK)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "direction must be RQ_HALF_PACK or RQ_HALF_UNPACK");
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, device_buf) != cudaSuccess || at.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "the buffer must be device memory");
    }
    RQ_TRY(set_device(s));
    return rq::half_copy(s, qubit, value, device_buf, direction == RQ_HALF_UNPACK ? 1 : 0);
}

int rq_state_negate_all_except(rq_state* s, uint64_t keep) {
    if (!s) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null state");
    RQ_TRY(set_device(s));
    return rq::negate_except(s, keep);
}

int rq_state_fidelity(rq_state* a, rq_state* b, double* out) {
    if (!a || !b || !out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (a->nq != b->nq) {
        *out = 0.0;
        return RQ_OK;
    }
    RQ_TRY(set_device(a));
    double re = 0, im = 0;
    RQ_TRY(rq::inner(a, b, &re, &im));
    *out = re * re + im * im;
    return RQ_OK;
}

int rq_state_download(rq_state* s, double* out) {
    if (!s || !out) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_TRY(set_device(s));
    size_t bytes = s->n * 2 * sizeof(double);
    if (s->prec == RQ_F64) {
        RQ_CUDA(cudaMemcpyAsync(out, s->amps, bytes, cudaMemcpyDeviceToHost, s->stream));
        return rq::sync_checked(s);
    }
    double* d = nullptr;
    RQ_CUDA(cudaMallocAsync((void**)&d, bytes, s->stream));
    int rc = rq::download_f64(s, d);
    cudaError_t e = cudaSuccess;
    if (rc == RQ_OK) e = cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, s->stream);
    cudaFreeAsync(d, s->stream);
    RQ_TRY(rc);
    RQ_CUDA(e);
    return rq::sync_checked(s);
}

int rq_state_upload(rq_state* s, const double* in) {
    if (!s || !in) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_TRY(set_device(s));
    size_t bytes = s->n * 2 * sizeof(double);
    if (s->prec == RQ_F64) {
        RQ_CUDA(cudaMemcpyAsync(s->amps, in, bytes, cudaMemcpyHostToDevice, s->stream));
        RQ_CUDA(cudaStreamSynchronize(s->stream));
        return RQ_OK;
    }
    double* d = nullptr;
    RQ_CUDA(cudaMallocAsync((void**)&d, bytes, s->stream));
    cudaError_t e = cudaMemcpyAsync(d, in, bytes, cudaMemcpyHostToDevice, s->stream);
    int rc = e == cudaSuccess ? rq::upload_f64(s, d) : rq::cuda_fail(e, "cudaMemcpyAsync");
    cudaFreeAsync(d, s->stream);
    RQ_TRY(rc);
    RQ_CUDA(cudaStreamSynchronize(s->stream));
    return RQ_OK;
}

}  // extern "C"
