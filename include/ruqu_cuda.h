/*
 * ruqu_cuda.h -- C-ABI boundary of the B200 state-vector engine.
 *
 * Every entry point here replaces one call of ruqu-core's dense state-vector
 * path (crate `ruqu-core`, files under crates/ruqu-core/src/) or one batched
 * loop of ruqu-algorithms' QAOA / VQE drivers.  The reference has no backend
 * trait for this path, so the boundary mirrors the `QuantumState` methods and
 * the `Simulator` calls one-for-one.  Plain pointers and sizes only; all
 * host arrays are owned by the caller and never retained after return.
 *
 * Threading: one rq_state owns one device buffer and one CUDA stream.  Calls
 * on one handle must be serialised by the caller (the reference state is a
 * single-owner `&mut self` value); distinct handles may be driven from
 * distinct threads.
 *
 * Errors: every function returns an rq_status.  Codes 1..5 mirror the
 * variants of `QuantumError` (crates/ruqu-core/src/error.rs:8-23);
 * rq_last_error_message() gives the formatted message of the last failure
 * on the calling thread.
 */
#ifndef RUQU_CUDA_H
#define RUQU_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RQ_API __attribute__((visibility("default")))
#else
#define RQ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- limits (crates/ruqu-core/src/state.rs:15, mixed_precision.rs:185) ---- */
#define RQ_MAX_QUBITS_F64 32u
#define RQ_MAX_QUBITS_F32 33u

/* ---- status codes (crates/ruqu-core/src/error.rs:8-23) ---- */
typedef enum rq_status {
    RQ_OK = 0,
    RQ_ERR_QUBIT_LIMIT_EXCEEDED = 1,    /* QuantumError::QubitLimitExceeded      */
    RQ_ERR_INVALID_QUBIT_INDEX = 2,     /* QuantumError::InvalidQubitIndex       */
    RQ_ERR_MEMORY_ALLOCATION = 3,       /* QuantumError::MemoryAllocationFailed  */
    RQ_ERR_INVALID_STATE_VECTOR = 4,    /* QuantumError::InvalidStateVector      */
    RQ_ERR_CIRCUIT = 5,                 /* QuantumError::CircuitError            */
    RQ_ERR_CUDA = 6,                    /* a CUDA runtime call failed            */
    RQ_ERR_TIMEOUT = 7,                 /* a bounded device-side wait expired    */
    RQ_ERR_INVALID_ARGUMENT = 8         /* null pointer / bad enum / bad size    */
} rq_status;

/* ---- amplitude precision ---- */
typedef enum rq_precision {
    RQ_F32 = 0,   /* interleaved complex float  (QuantumStateF32, mixed_precision.rs:193) */
    RQ_F64 = 1    /* interleaved complex double (QuantumState, state.rs:18)               */
} rq_precision;

/* ---- gate kinds, in the order of `enum Gate` (crates/ruqu-core/src/gate.rs:8-36) ---- */
typedef enum rq_gate_kind {
    RQ_GATE_H = 0,
    RQ_GATE_X = 1,
    RQ_GATE_Y = 2,
    RQ_GATE_Z = 3,
    RQ_GATE_S = 4,
    RQ_GATE_SDG = 5,
    RQ_GATE_T = 6,
    RQ_GATE_TDG = 7,
    RQ_GATE_RX = 8,
    RQ_GATE_RY = 9,
    RQ_GATE_RZ = 10,
    RQ_GATE_PHASE = 11,
    RQ_GATE_CNOT = 12,       /* q0 = control, q1 = target */
    RQ_GATE_CZ = 13,
    RQ_GATE_SWAP = 14,
    RQ_GATE_RZZ = 15,
    RQ_GATE_MEASURE = 16,
    RQ_GATE_RESET = 17,
    RQ_GATE_BARRIER = 18,
    RQ_GATE_UNITARY1Q = 19   /* m[] holds the 2x2 matrix */
} rq_gate_kind;

/* One gate, plain old data (replaces `Gate`, gate.rs:8-36). */
typedef struct rq_gate {
    int32_t  kind;      /* rq_gate_kind                                            */
    uint32_t q0;        /* the qubit (1q gates) / first qubit (2q gates)           */
    uint32_t q1;        /* second qubit of 2q gates, ignored otherwise             */
    uint32_t pad;       /* zero                                                    */
    double   angle;     /* Rx/Ry/Rz/Phase/Rzz angle in radians                     */
    double   m[8];      /* UNITARY1Q: m00 m01 m10 m11 as (re,im) pairs, row-major  */
} rq_gate;

/* One measurement result (replaces `MeasurementOutcome`, types.rs:230-235). */
typedef struct rq_measurement {
    uint32_t qubit;
    int32_t  result;       /* 1 = measured |1> */
    double   probability;  /* probability of the observed branch */
} rq_measurement;

/* Pauli factors (replaces `PauliOp`, types.rs:190-197). */
typedef enum rq_pauli { RQ_PAULI_I = 0, RQ_PAULI_X = 1, RQ_PAULI_Y = 2, RQ_PAULI_Z = 3 } rq_pauli;

typedef struct rq_pauli_op {
    uint32_t qubit;
    int32_t  op;           /* rq_pauli */
} rq_pauli_op;

/* Execution modes for rq_state_apply (the reference always runs one pass per gate). */
typedef enum rq_exec_mode {
    RQ_EXEC_AUTO = 0,      /* autotuned choice (default) */
    RQ_EXEC_PER_GATE = 1,  /* one kernel per gate: the unfused path              */
    RQ_EXEC_SWEEP = 2,     /* register/shared-memory tiled multi-gate sweeps     */
    RQ_EXEC_SWEEP_TC = 3,  /* sweeps whose per-phase gate runs are fused into dense
                              32x32 unitaries applied on the tensor cores as
                              3xTF32 MMAs (complex f32 states, >= 12 qubits)     */
    RQ_EXEC_SWEEP_TC_FAST = 4, /* as RQ_EXEC_SWEEP_TC with one TF32 MMA pass
                                  (10-bit operand mantissas)                     */
    RQ_EXEC_SWEEP_TC16 = 5     /* as RQ_EXEC_SWEEP_TC with the dense ops as three
                                  FP16 MMA passes (hi*hi + hi*lo + lo*hi of
                                  per-tile-scaled amplitudes and 2^14-scaled
                                  unitaries, FP32 accumulation): FP32-level
                                  accuracy at twice the TF32 tensor rate; a list
                                  with a non-unitary UNITARY1Q matrix runs as
                                  RQ_EXEC_SWEEP_TC                               */
} rq_exec_mode;

typedef struct rq_state rq_state;   /* opaque: device-resident amplitudes */
typedef struct rq_plan rq_plan;     /* opaque: a gate list prepared for one state shape */

/* What a prepared plan launches (filled by rq_plan_get_stats). */
typedef struct rq_plan_stats {
    uint64_t gates;       /* unitary gates in the plan                          */
    uint64_t launches;    /* kernel launches per execution                      */
    uint64_t sweeps;      /* full passes over the state (sweep mode)            */
    uint64_t phases;      /* register phases summed over all sweeps             */
    uint64_t ops;         /* device ops after 1-qubit fusion                    */
    uint64_t hbm_bytes;   /* algorithmic HBM bytes per execution                */
    uint64_t dense_ops;   /* dense 32x32 unitaries on the tensor cores          */
    uint64_t exec_mode;   /* rq_exec_mode the plan runs (RQ_EXEC_AUTO resolved)  */
    uint64_t local_qubits;/* qubits per tile of a sweep (0: per-gate)            */
} rq_plan_stats;

/* ------------------------------------------------------------------------ */
/* errors / library                                                          */
/* ------------------------------------------------------------------------ */

/* Message of the last failing call on this thread ("" if none). */
RQ_API const char* rq_last_error_message(void);

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
RQ_API int32_t rq_version(void);

/* One draw of the documented uniform stream (Philox4x32-10, Salmon et al.,
 * SC'11): u in [0,1) with 53 random bits.  Draw `index` of `stream` under
 * key `seed`.  Stream 0 feeds measurements; shot s of a run_shots call with
 * base seed b uses key b+s (wrapping), mirroring simulator.rs:124-130. */
RQ_API double rq_uniform(uint64_t seed, uint32_t stream, uint64_t index);

/* Select the CUDA device used by states created afterwards on this thread. */
RQ_API int rq_device_set(int32_t device);
RQ_API int rq_device_count(int32_t* out);

/* ------------------------------------------------------------------------ */
/* state lifetime (state.rs:31-96, mixed_precision.rs:214-280)               */
/* ------------------------------------------------------------------------ */

/* QuantumState::new / new_with_seed (seeded != 0).  |0...0>.  0 qubits is a
 * CircuitError for both (state.rs:32-36 checks it in `new` only; the seeded
 * constructor would build a 1-amplitude state -- we reject it in both). */
RQ_API int rq_state_create(uint32_t num_qubits, int32_t precision, uint64_t seed,
                    int32_t seeded, rq_state** out);

/* QuantumState::from_amplitudes (state.rs:75-96): `len` complex values given
 * as 2*len interleaved doubles; len must equal 2^num_qubits. */
RQ_API int rq_state_from_amplitudes(const double* interleaved, uint64_t len,
                             uint32_t num_qubits, int32_t precision,
                             uint64_t seed, rq_state** out);

RQ_API int rq_state_destroy(rq_state* s);

/* Back to |0...0>, measurement stream rewound to draw 0 of the same seed.
 * Stream-ordered: returns once the init kernel is queued. */
RQ_API int rq_state_reset(rq_state* s);

RQ_API int rq_state_num_qubits(const rq_state* s, uint32_t* out);
RQ_API int rq_state_precision(const rq_state* s, int32_t* out);

/* Device pointer of the amplitudes (interleaved complex) and its stream, for
 * zero-copy interop; valid until rq_state_destroy. */
RQ_API int rq_state_device_ptr(const rq_state* s, void** out_ptr, void** out_stream);

/* Block the host until all work queued on the state's stream is done. */
RQ_API int rq_state_synchronize(rq_state* s);

/* Test hook, no counterpart in the reference: the number of polls a
 * tensor-core kernel (the sweeps of RQ_EXEC_SWEEP_TC / _FAST / _TC16 and the
 * BF16 GEMM) makes on an mbarrier before its wait counts as expired, on the
 * current device; RQ_WAIT_LIMIT_DEFAULT restores the default.  With 0 polls
 * the waits run out at once: the kernel sets its error flag, waits (with the
 * default limit) for its copies and MMAs in flight, frees its tensor memory
 * and returns; the next read-back of the state (rq_state_synchronize,
 * rq_state_download, an expectation, probabilities or samples) -- or the
 * GEMM call itself -- reports RQ_ERR_TIMEOUT and clears the flag, and the
 * state's handle stays usable (its amplitudes are not: reset or upload). */
#define RQ_WAIT_LIMIT_DEFAULT 0xFFFFFFFFu
RQ_API int rq_debug_set_wait_limit(uint32_t polls);

/* ------------------------------------------------------------------------ */
/* gates (state.rs:158-276)                                                  */
/* ------------------------------------------------------------------------ */

/* Apply `n` gates in order (QuantumState::apply_gate in a loop, as
 * Simulator::run_with_config does, simulator.rs:69-79).  Validation happens
 * for the whole list before anything runs; an invalid gate returns its error
 * and leaves the state untouched.  Measure/Reset outcomes are written to
 * `out` (capacity `cap`); their count goes to *nout (out may be NULL when
 * the list has no Measure/Reset). */
RQ_API int rq_state_apply(rq_state* s, const rq_gate* gates, uint64_t n,
                   rq_measurement* out, uint64_t cap, uint64_t* nout);

/* Same, with an explicit execution mode (rq_exec_mode). */
RQ_API int rq_state_apply_mode(rq_state* s, const rq_gate* gates, uint64_t n,
                        int32_t mode, rq_measurement* out, uint64_t cap,
                        uint64_t* nout);

/* NoiseModel (types.rs:249-263). */
typedef struct rq_noise_model {
    double depolarizing_rate;
    double bit_flip_rate;
    double phase_flip_rate;
} rq_noise_model;

/* rq_state_apply with a noise model: the gate loop of Simulator::run_with_config
 * when config.noise is set (simulator.rs:67-78).  After every gate with qubits
 * (Measure and Reset included, Barrier not), each of its qubits in order draws
 * from the state's measurement stream as apply_noise does (simulator.rs:177-221):
 * a depolarising draw r (< rate: a second draw picks X / Y / Z by thirds), a
 * bit-flip draw (< rate: X), a phase-flip draw (< rate: Z); a channel whose rate
 * is 0 draws nothing.  Measurements keep their place in the same stream.  The
 * chosen Paulis are applied on the device with the rest of the list. */
RQ_API int rq_state_apply_noisy(rq_state* s, const rq_gate* gates, uint64_t n,
                                const rq_noise_model* noise, rq_measurement* out, uint64_t cap,
                                uint64_t* nout);

/* apply_single_qubit_gate (state.rs:214-229): m = 8 doubles, (re,im) pairs. */
RQ_API int rq_state_apply_1q_matrix(rq_state* s, uint32_t qubit, const double* m);

/* apply_two_qubit_gate (state.rs:238-276): m = 32 doubles, 4x4 row-major,
 * row/column index = q1_bit*2 + q2_bit. */
RQ_API int rq_state_apply_2q_matrix(rq_state* s, uint32_t q1, uint32_t q2,
                             const double* m);

/* Prepared plans: the gate list of Simulator::run_with_config
 * (simulator.rs:69-79) planned once for states of s's qubit count and
 * precision, with its tables uploaded to the device.  rq_plan_execute only
 * launches kernels on the state's stream (no host sync, no allocation), so a
 * plan can be replayed cheaply or captured in a CUDA graph.  Unitary gates
 * only (Measure / Reset are rejected with RQ_ERR_CIRCUIT; Barrier is
 * dropped).  mode: rq_exec_mode. */
RQ_API int rq_plan_create(const rq_state* s, const rq_gate* gates, uint64_t n,
                          int32_t mode, rq_plan** out);
RQ_API int rq_plan_execute(rq_state* s, const rq_plan* p);

/* As rq_plan_create with the tile size of a tensor-core sweep chosen by the caller (the
 * autotuner of RQ_EXEC_AUTO picks among these itself): local_qubits 12 or 13 for
 * RQ_EXEC_SWEEP_TC / _TC_FAST, 12, 13 or 14 for RQ_EXEC_SWEEP_TC16 (12: four 128-thread CTAs
 * per SM, more sweeps; 13: two 256-thread CTAs per SM; 14: one 512-thread CTA per SM, fewer
 * sweeps), complex f32 states only; 0 = the default.  No counterpart in the reference. */
RQ_API int rq_plan_create_tiled(const rq_state* s, const rq_gate* gates, uint64_t n, int32_t mode,
                                uint32_t local_qubits, rq_plan** out);

/* New gate values for a prepared plan: `gates` must have the plan's gate kinds and
 * qubits (barriers aside) and may change any angle or matrix.  No counterpart in the
 * reference (whose drivers rebuild the circuit for every evaluation, qaoa.rs:232 and
 * vqe.rs:129); this is what makes those evaluations cheap here: the plan's sweeps and
 * phases are kept, the fused matrices are re-derived on the host and the tensor-core
 * operand images rebuilt on the GPU, in stream order on s's stream (after every earlier
 * launch of the plan, on any stream).  RQ_ERR_CIRCUIT when the structure differs (the
 * plan is then unchanged).  rq_state_apply does the same by itself for gate lists that
 * repeat the structure of a recently applied list. */
RQ_API int rq_plan_update(rq_state* s, rq_plan* p, const rq_gate* gates, uint64_t n);
RQ_API int rq_plan_get_stats(const rq_plan* p, rq_plan_stats* out);
RQ_API int rq_plan_destroy(rq_plan* p);

/* ------------------------------------------------------------------------ */
/* noise channels (noise.rs:151-280)                                         */
/* One quantum-trajectory step of a single-qubit noise channel given by its Kraus
 * operators (kraus: nk row-major 2x2 matrices, 8 doubles each as (re, im) pairs, the
 * sets of depolarizing_kraus / amplitude_damping_kraus / phase_damping_kraus /
 * thermal_relaxation_kraus, noise.rs:166-280).  The reference builds these sets but no
 * caller applies them to a state; here, with rho the qubit's reduced density matrix,
 * operator k is chosen with probability p_k = tr(K_k rho K_k^dagger) / sum_j p_j using
 * the next uniform of the state's measurement stream (the draw a measurement would
 * take), and the state becomes K_k |psi> / sqrt(p_k) (its norm kept).  Averaged over
 * trajectories this is the channel.  *chosen = k, *probability = its p_k (either may be
 * NULL).  Two device passes: the reduction of <I>, <Z_q>, <X_q>, <Y_q> and the 2x2
 * update.  RQ_ERR_INVALID_STATE_VECTOR if every p_k is 0. */
#define RQ_KRAUS_MAX 16u
RQ_API int rq_state_apply_kraus(rq_state* s, uint32_t q, const double* kraus, uint32_t nk,
                                int32_t* chosen, double* probability);

/* ------------------------------------------------------------------------ */
/* measurement (state.rs:288-352)                                            */

RQ_API int rq_state_measure(rq_state* s, uint32_t qubit, rq_measurement* out);
RQ_API int rq_state_measure_all(rq_state* s, rq_measurement* out /* num_qubits */);
RQ_API int rq_state_reset_qubit(rq_state* s, uint32_t qubit);

/* Shot sampling without collapse.  Reproduces, shot by shot, the outcome of
 * Simulator::run_shots (simulator.rs:107-147): shot s measures `qubits` in
 * the given order with draws 0,1,2,... of key base_seed+s, outcome 1 iff
 * u >= P(qubit=0 | earlier outcomes).  out_bits[s] has bit q set iff qubit q
 * was measured as 1.  The state is not modified. */
RQ_API int rq_state_sample(rq_state* s, const uint32_t* qubits, uint32_t nqubits,
                    uint64_t base_seed, uint64_t shots, uint64_t* out_bits);

/* The prefix tree rq_state_sample walks, kept with the state for lookups: the qubits
 * ordered as `qubits` lists them (first appearance; the qubits not listed after them),
 * level L (0 <= L <= num_qubits) holds 2^L FP64 sums of |a_i|^2, entry j over the
 * amplitudes whose first L ordered qubits take the bits of j (bit k of j = qubit k of
 * that order); level 0 is the squared norm, level num_qubits the |a_i|^2 themselves.
 * A snapshot of the amplitudes at build time (level num_qubits reads them live): build
 * again after the state changes.  rq_state_sample replaces it with its own tree.
 * A rank of a state split over several GPUs samples or measures through these sums: its
 * share of every conditional probability of the shot walk (simulator.rs:107-147) is one
 * lookup, and the ranks add their shares (ruqu_b200/distributed.py). */
RQ_API int rq_state_tree_build(rq_state* s, const uint32_t* qubits, uint32_t nqubits);
/* out[i] = entry index[i] of level `level` (host arrays; index[i] < 2^level). */
RQ_API int rq_state_tree_lookup(rq_state* s, uint32_t level, const uint64_t* index, uint64_t count,
                                double* out);

/* ------------------------------------------------------------------------ */
/* reductions (state.rs:123-137, 362-435)                                    */
/* ------------------------------------------------------------------------ */

/* |a_i|^2 for all i into host memory (2^n doubles). */
RQ_API int rq_state_probabilities(rq_state* s, double* out);

RQ_API int rq_state_probability_of_qubit(rq_state* s, uint32_t qubit, double* out);

/* expectation_value(PauliString) (state.rs:362-400), FP64 accumulation. */
RQ_API int rq_state_expectation_value(rq_state* s, const rq_pauli_op* ops,
                               uint32_t nops, double* out);

/* Many Pauli strings in one call: string k is ops[offsets[k] .. offsets[k+1]).
 * out[k] = <P_k>. */
RQ_API int rq_state_expectation_batch(rq_state* s, const rq_pauli_op* ops,
                               const uint32_t* offsets, uint32_t nstrings,
                               double* out);

/* expectation_hamiltonian (state.rs:403-408): sum_k coeffs[k] <P_k>. */
RQ_API int rq_state_expectation_hamiltonian(rq_state* s, const double* coeffs,
                                     const rq_pauli_op* ops,
                                     const uint32_t* offsets, uint32_t nterms,
                                     double* out);

/* Allocation-free variant of rq_state_expectation_batch.  No counterpart in
 * the reference.  For callers that must not allocate device memory -- for
 * example code that runs with a fixed memory budget already handed out, or a
 * process whose allocator is owned by another framework -- this entry point
 * takes the amplitudes as a caller-owned device pointer (interleaved complex,
 * 2^num_qubits values of `precision`) and keeps its reduction partials in one
 * fixed static device array of RQ_NOALLOC_SCRATCH_DOUBLES doubles (~1.1 MB per
 * GPU that loads the library, held until the process exits).
 *   - at most RQ_NOALLOC_MAX_STRINGS strings per call; more is rejected with
 *     RQ_ERR_INVALID_ARGUMENT and nothing runs;
 *   - the first call on a device looks up the scratch address for that device
 *     (with the device current), and so does the first call after the
 *     device's context was re-created (cudaDeviceReset); make that first call
 *     before any stream capture;
 *   - every call shares the one scratch array and keeps nothing from earlier
 *     calls (each call writes every partial it reads), so calls that overlap
 *     on the GPU (other streams, other host threads) race: serialise them;
 *   - runs on `stream` (a cudaStream_t, NULL = the legacy default stream) on
 *     the current device; it blocks the host: it copies the sums back and
 *     synchronises `stream` before it returns with the results in out[];
 *   - a NULL `ops` with a non-empty string is rejected (RQ_ERR_INVALID_ARGUMENT).
 * It calls no cudaMalloc / cudaFree and no allocating library routine. */
#define RQ_NOALLOC_MAX_STRINGS 128u
#define RQ_NOALLOC_MAX_BLOCKS 1024u
#define RQ_NOALLOC_SCRATCH_DOUBLES ((RQ_NOALLOC_MAX_STRINGS + 1u) * RQ_NOALLOC_MAX_BLOCKS)
RQ_API int rq_expectation_batch_noalloc(const void* device_amps, uint32_t num_qubits,
                                        int32_t precision, const rq_pauli_op* ops,
                                        const uint32_t* offsets, uint32_t nstrings,
                                        double* out, void* stream);

RQ_API int rq_state_norm_sq(rq_state* s, double* out);
RQ_API int rq_state_normalize(rq_state* s);                         /* state.rs:415-423 */
RQ_API int rq_state_fidelity(rq_state* a, rq_state* b, double* out); /* state.rs:426-435 */

/* The host amplitude edits of run_grover (grover.rs:128-153, through
 * amplitudes_mut) as device passes, so the state stays on the device.
 * rq_state_negate_amplitudes: amps[i] = -amps[i] for every listed index (the
 * oracle step, grover.rs:128-139); an index listed twice is negated twice, as
 * the reference's loop does; an index >= 2^n is rejected (run_grover asserts,
 * grover.rs:103-111) and nothing changes.
 * rq_state_negate_all_except: amps[i] = -amps[i] for every i != keep (the
 * diffuser's 2|0><0| - I between the Hadamard layers with keep = 0,
 * grover.rs:144-153).  No reference counterpart as functions. */
RQ_API int rq_state_negate_amplitudes(rq_state* s, const uint64_t* indices, uint64_t count);
RQ_API int rq_state_negate_all_except(rq_state* s, uint64_t keep);

/* A state split over ranks by its top qubits (a distributed state) makes a global
 * qubit local by swapping it with a local qubit: each rank sends the half of its
 * amplitudes whose local bit `qubit` differs from its own bit of the global qubit and
 * receives the partner's half into the same places.  rq_state_half_copy copies the
 * half with bit `qubit` == `value` (2^(n-1) amplitudes of the state's precision, in
 * the order of the other bits) into a contiguous device buffer (RQ_HALF_PACK) or back
 * from one (RQ_HALF_UNPACK), on the state's stream.  No reference counterpart (the
 * reference has no distributed state). */
#define RQ_HALF_PACK 0
#define RQ_HALF_UNPACK 1
RQ_API int rq_state_half_copy(rq_state* s, uint32_t qubit, uint32_t value, void* device_buf,
                              int32_t direction);

/* ------------------------------------------------------------------------ */
/* batched QAOA-MaxCut (qaoa.rs:125-201 over many graphs / parameter sets)    */
/* ------------------------------------------------------------------------ */

typedef struct rq_qaoa_batch rq_qaoa_batch;

/* `ninst` simple unweighted graphs (unit weights, as the MaxCut instances of
 * qaoa.rs:59-66 `Graph::unweighted`): graph k has num_nodes[k] vertices
 * (7..30 for f32 states, 6..30 for f64) and the edges
 * edges[2e], edges[2e+1] for e in [edge_offsets[k], edge_offsets[k+1]).
 * p = QAOA depth.  The graphs and the planned sweep programs stay on the GPU. */
RQ_API int rq_qaoa_batch_create(uint32_t ninst, const uint32_t* num_nodes,
                                const uint32_t* edge_offsets, const uint32_t* edges,
                                uint32_t p, int32_t precision, rq_qaoa_batch** out);

/* Evaluate ninst*nsets circuits: circuit c = inst*nsets + set uses
 * gammas[c*p .. c*p+p) and betas[c*p .. c*p+p) and the graph of inst.  Each
 * is the circuit of build_qaoa_circuit; energies[c] = its expected cut
 * sum_edges (1 - <Z_i Z_j>)/2 (evaluate_qaoa_cost), accumulated in FP64.
 * With shots > 0, shot s of circuit c measures all qubits in order with draws
 * 0..n-1 of key base_seed + (c << 32) + s (the run_shots semantics of
 * simulator.rs:107-147 with that seed), and best_bits[c] / best_cut[c] are
 * the sampled bitstring with the highest cut (lowest shot index on ties). */
RQ_API int rq_qaoa_batch_run(rq_qaoa_batch* b, uint32_t nsets, const double* gammas,
                             const double* betas, double* energies, uint32_t shots,
                             uint64_t base_seed, uint64_t* best_bits, uint32_t* best_cut);

/* Gradient rules of rq_qaoa_batch_optimize.
 * RQ_QAOA_GRAD_ADJOINT: exact dE/dgamma_l, dE/dbeta_l by one backward pass
 *   (2 Im <lambda|G|psi> per gate generator G, lambda = C psi carried back).
 * RQ_QAOA_GRAD_SHIFT: the rule of run_qaoa (qaoa.rs:275-297), (E(theta_k +
 *   pi/2) - E(theta_k - pi/2)) / 2 with the shift applied to a whole layer's
 *   angle.  For unit edge weights it is zero up to rounding: shifting every
 *   Rzz(2 gamma) of a layer by pi/2 multiplies the state by a Pauli string
 *   (up to phase) that cancels between the two evaluations, and likewise for
 *   the Rx(2 beta) of a layer.  Kept to reproduce the reference's rule. */
#define RQ_QAOA_GRAD_ADJOINT 0
#define RQ_QAOA_GRAD_SHIFT 1

/* Energies and exact gradients of ninst circuits (one per graph):
 * gammas / betas are ninst x p; energies[i] as rq_qaoa_batch_run;
 * gradients[i*2p + l] = dE/dgamma_l, gradients[i*2p + p + l] = dE/dbeta_l,
 * reduced in FP64.  No reference counterpart (run_qaoa only has the shift
 * rule). */
RQ_API int rq_qaoa_batch_gradient(rq_qaoa_batch* b, const double* gammas, const double* betas,
                                  double* energies, double* gradients);

/* Batched run_qaoa (qaoa.rs:217-308) with Adam: for up to `steps` steps every
 * instance takes its gradient by `gradient` (RQ_QAOA_GRAD_*) and Adam
 * (0.9, 0.999, 1e-8, learning rate lr) climbs the expected cut; parameters,
 * moments and updates are FP64 on the device.  gammas / betas (ninst x p) are
 * the start and receive the result.  With a target (ninst values) an instance
 * stops once its energy reaches target * (1 - rtol) and leaves the following
 * steps' launches; steps_taken[i] = the step at which it did (or `steps`).
 * energies[i] = energy at the returned angles (at the stop). */
RQ_API int rq_qaoa_batch_optimize(rq_qaoa_batch* b, uint32_t steps, double lr, double* gammas, double* betas,
                                  const double* target, double rtol, int32_t gradient, double* energies,
                                  uint32_t* steps_taken);

/* As rq_qaoa_batch_optimize with exact gradients, but each step is a preconditioned
 * ascent step theta += alpha_i * P_i * grad E with the caller's 2p x 2p matrix P_i per
 * instance (precond: ninst x 2p x 2p, row-major, theta = (gammas, betas)), e.g. a learned
 * -H^-1 of the family's energy landscape; alpha_i starts at alpha and halves whenever the
 * instance's energy fell since its previous step.  No reference counterpart. */
RQ_API int rq_qaoa_batch_optimize_precond(rq_qaoa_batch* b, uint32_t steps, const double* precond, double alpha,
                                          double* gammas, double* betas, const double* target, double rtol,
                                          double* energies, uint32_t* steps_taken);

/* The convergence rule of run_qaoa (qaoa.rs:266-269) for both optimizers of this batch:
 * an instance stops (as when it meets its target) once its energy changed by less than
 * tol since the previous step.  tol = 0 (the default) turns it off; run_qaoa uses 1e-6. */
RQ_API int rq_qaoa_batch_set_convergence(rq_qaoa_batch* b, double tol);

/* Final amplitudes of one circuit of the last run (2^n interleaved doubles);
 * only circuits of the last memory wave of that run are still held. */
RQ_API int rq_qaoa_batch_state(rq_qaoa_batch* b, uint64_t circuit, double* interleaved);

/* Device time of the last run (CUDA events around all of its kernels), ms. */
RQ_API int rq_qaoa_batch_last_ms(const rq_qaoa_batch* b, float* ms);
/* Device time and algorithmic work of the last rq_qaoa_batch_run / _gradient, by kernel
 * kind (no counterpart in the reference): out6 = {sweep HBM bytes, sweep ms, sampling
 * bytes, sampling ms, adjoint bytes, adjoint ms}.  Bytes are algorithmic: per circuit
 * and sweep, S written by an initialising sweep and 2S for a read and a write otherwise
 * (two states in the adjoint pass), and per sampled circuit S + 2^n x 16 bytes for the
 * prefix tree; times are CUDA events around each class's launches. */
RQ_API int rq_qaoa_batch_last_profile(const rq_qaoa_batch* b, double* out6);

/* CUDA graphs of the batched runs (rq_qaoa_batch_run / _gradient, rq_vqe_batch_run): the
 * first run of a shape (sizes, gradient mode, shots and seed, buffers) launches its kernels
 * one by one and is the one the profile describes; the next run of the same shape captures
 * the same kernels into a graph and launches it, later runs replay it (one launch per run;
 * the angles and parameters are uploaded before it, the results read after it).  Results
 * are those of the plain launches.  On by default (off with RUQU_NO_GRAPHS=1 in the
 * environment).  *replayed = 1 if the last run launched the graph, *kernels = the kernels
 * in the captured graph. */
RQ_API int rq_qaoa_batch_set_graphs(rq_qaoa_batch* b, int32_t enable);
RQ_API int rq_qaoa_batch_last_graph(const rq_qaoa_batch* b, int32_t* replayed, uint64_t* kernels);

/* Upper bound of state memory per wave (default 24 GiB). */
RQ_API int rq_qaoa_batch_set_state_budget(rq_qaoa_batch* b, uint64_t bytes);

RQ_API int rq_qaoa_batch_destroy(rq_qaoa_batch* b);

/* ------------------------------------------------------------------------ */
/* batched VQE (vqe.rs:122-216 over many parameter sets)                     */
/* ------------------------------------------------------------------------ */

typedef struct rq_vqe_batch rq_vqe_batch;

/* Hardware-efficient ansatz on num_qubits qubits, `depth` layers of "Ry(theta)
 * on every qubit, then CZ(q, q+1) for q = 0..n-2" (num_qubits*depth
 * parameters, layer-major), and the Hamiltonian sum_k coeffs[k] P_k with
 * P_k = ops[offsets[k] .. offsets[k+1]) (types.rs:218-228). */
RQ_API int rq_vqe_batch_create(uint32_t num_qubits, uint32_t depth, const double* coeffs,
                               const rq_pauli_op* ops, const uint32_t* offsets, uint32_t nterms,
                               int32_t precision, rq_vqe_batch** out);

/* Gradient modes of rq_vqe_batch_run.
 * RQ_VQE_GRAD_SHIFT: gradients[s*P + k] = (E(theta_k + pi/2) - E(theta_k - pi/2)) / 2,
 *   the parameter-shift rule of run_vqe (vqe.rs:186-198): 1 + 2P circuits per set.
 * RQ_VQE_GRAD_ADJOINT: the same derivative (the shift rule is exact for Ry) by one
 *   backward pass per set: lambda = H psi, then psi and lambda run back through the
 *   ansatz and every Ry(theta_k) = exp(-i theta_k Y/2) contributes Im <lambda|Y|psi>.
 *   No reference counterpart (run_vqe only has the shift rule). */
#define RQ_VQE_GRAD_NONE 0
#define RQ_VQE_GRAD_SHIFT 1
#define RQ_VQE_GRAD_ADJOINT 2

/* energies[s] = <psi(params_s)|H|psi(params_s)> (evaluate_energy, vqe.rs:122-131)
 * for s < nsets, params_s = params[s*P .. s*P+P); with_gradient (RQ_VQE_GRAD_*)
 * selects whether and how gradients[s*P + k] = dE/dtheta_k is computed.  All
 * circuits run on the device in waves; energies and gradients accumulate in FP64. */
RQ_API int rq_vqe_batch_run(rq_vqe_batch* b, uint32_t nsets, const double* params,
                            int32_t with_gradient, double* energies, double* gradients);

RQ_API int rq_vqe_batch_last_ms(const rq_vqe_batch* b, float* ms);
/* As rq_qaoa_batch_last_profile for the last rq_vqe_batch_run: {evolution sweep bytes,
 * evolution ms, energy-pass floating-point operations (8 per string and amplitude),
 * energy ms, adjoint bytes (the H pass and the backward program over two states),
 * adjoint ms}.  The waves are sized to stay in L2, so the sweep bytes are mostly L2
 * traffic.  No counterpart in the reference. */
RQ_API int rq_vqe_batch_last_profile(const rq_vqe_batch* b, double* out6);
/* As rq_qaoa_batch_set_graphs / _last_graph for rq_vqe_batch_run. */
RQ_API int rq_vqe_batch_set_graphs(rq_vqe_batch* b, int32_t enable);
RQ_API int rq_vqe_batch_last_graph(const rq_vqe_batch* b, int32_t* replayed, uint64_t* kernels);
RQ_API int rq_vqe_batch_destroy(rq_vqe_batch* b);

/* ------------------------------------------------------------------------ */
/* BF16 tensor-core GEMM and the QAOA warm-start MLP (no reference            */
/* counterpart: the reference starts QAOA from gamma = beta = 0.5,            */
/* qaoa.rs:221-222)                                                           */
/* ------------------------------------------------------------------------ */

/* C (f32, M x N, row-major) = A (bf16 bits, M x K) * B (bf16 bits, N x K)^T on
 * the tcgen05 tensor cores, FP32 accumulation.  Any M, N >= 1; K a positive
 * multiple of 16. */
RQ_API int rq_gemm_bf16(const uint16_t* A, const uint16_t* B, int32_t M, int32_t N, int32_t K, float* C);

typedef struct rq_mlp rq_mlp;

/* MLP in -> h1 -> h2 -> out with ReLU after both hidden layers; FP32 master
 * parameters laid out flat as W1 [h1 x in], b1 [h1], W2 [h2 x h1], b2 [h2],
 * W3 [out x h2], b3 [out] (weights row-major, one row per output unit);
 * BF16 copies feed the tensor-core GEMMs; He-uniform init from Philox stream 6
 * under `seed`.  h1, h2 multiples of 16. */
RQ_API int rq_mlp_create(int32_t in, int32_t h1, int32_t h2, int32_t out, uint64_t seed, rq_mlp** res);
RQ_API int rq_mlp_destroy(rq_mlp* m);
RQ_API int rq_mlp_num_params(const rq_mlp* m, int64_t* n);
RQ_API int rq_mlp_get_params(rq_mlp* m, float* params);
RQ_API int rq_mlp_set_params(rq_mlp* m, const float* params);   /* also resets Adam */
/* y (B x out) = MLP(x (B x in)), host buffers. */
RQ_API int rq_mlp_forward(rq_mlp* m, const float* x, int32_t B, float* y);
/* Mean-squared-error loss against t (B x out) and its gradient w.r.t. every
 * parameter (flat, parameter layout). */
RQ_API int rq_mlp_gradients(rq_mlp* m, const float* x, const float* t, int32_t B, float* loss, float* grads);
/* `steps` Adam steps (lr, 0.9, 0.999, 1e-8) on minibatches of B rows taken in
 * order (wrapping) from x (n x in), t (n x out); last step's loss out. */
RQ_API int rq_mlp_train(rq_mlp* m, const float* x, const float* t, int32_t n, int32_t B, int32_t steps, float lr,
                        float* last_loss);

/* ------------------------------------------------------------------------ */
/* host transfer (state_vector / amplitudes_mut / from_amplitudes)           */
/* ------------------------------------------------------------------------ */

/* 2^n complex values as 2^(n+1) interleaved doubles. */
RQ_API int rq_state_download(rq_state* s, double* interleaved);
RQ_API int rq_state_upload(rq_state* s, const double* interleaved);

#ifdef __cplusplus
}
#endif

#endif /* RUQU_CUDA_H */
