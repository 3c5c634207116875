/*
 * ket_sv.h -- C ABI of the B200 dense statevector engine for ket.
 *
 * The engine replaces the statevector path of the ket TypeScript library
 * (dmvjs/ket): the sparse Map<bigint,Complex> kernels of src/statevector.ts
 * driven by simulatePure (src/circuit.ts:143-161) and the read-outs that
 * consume its result (run / exactProbs / statevector / amplitude /
 * probability / marginals / expectation, and vqe / gradient / minimize in
 * src/algorithms.ts).  Each entry point below names the reference interface
 * it replaces.
 *
 * Conventions (identical to the reference):
 *   - basis index bit q is qubit q (q0 = LSB, src/statevector.ts:4-5);
 *   - in every multi-qubit matrix the FIRST listed qubit is the MOST
 *     significant bit of the local index (src/statevector.ts:32,107-108,237);
 *   - bitstrings are parsed/printed by the host (q0 leftmost); this ABI only
 *     sees integer indices.
 *
 * Threading: calls on one ket_ctx are serialised by the caller (the JS
 * caller is single threaded, like the reference).  Every call that returns
 * data blocks until the data is on the host.  Distinct contexts are
 * independent.  No entry point keeps a caller pointer after it returns.
 *
 * Errors: every function returns a ket_status; ket_last_error() returns a
 * thread-local message for the last failure on the calling thread.
 */
#ifndef KET_SV_H
#define KET_SV_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define KET_API __attribute__((visibility("default")))
#else
#define KET_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define KET_SV_ABI_VERSION 1

typedef enum ket_status {
  KET_OK = 0,
  KET_ERR_RANGE = 1,       /* qubit index out of range: the reference throws RangeError (circuit.ts:1114-1117) */
  KET_ERR_TYPE = 2,        /* control == target, bad matrix shape, bad argument: TypeError (circuit.ts:1118-1145) */
  KET_ERR_OOM = 3,         /* device allocation failed */
  KET_ERR_CUDA = 4,        /* a CUDA runtime call failed */
  KET_ERR_TIMEOUT = 5,     /* a bounded device wait ran out (status word set by the kernel) */
  KET_ERR_UNSUPPORTED = 6  /* a valid request the engine does not implement */
} ket_status;

typedef enum ket_precision { KET_C128 = 0, KET_C64 = 1 } ket_precision;

/* Op kinds: the FlatOp union of src/circuit.ts:20-47.  measure / reset / if
 * are accepted only by ket_run_shots (the pure path never sees them,
 * src/circuit.ts:1432-1438). */
typedef enum ket_op_kind {
  KET_OP_SINGLE = 0,      /* q[0];            2x2 matrix   (applySingle, statevector.ts:47)      */
  KET_OP_CNOT = 1,        /* q = {c, t}                    (applyCNOT, :70)                      */
  KET_OP_SWAP = 2,        /* q = {a, b}                    (applySWAP, :85)                      */
  KET_OP_TWO = 3,         /* q = {a, b};      4x4, a = MSB (applyTwo, :110)                      */
  KET_OP_CONTROLLED = 4,  /* q = {c, t};      2x2          (applyControlled, :212)               */
  KET_OP_TOFFOLI = 5,     /* q = {c1, c2, t}               (applyToffoli, :138)                  */
  KET_OP_CSWAP = 6,       /* q = {c, a, b}                 (applyCSwap, :153)                    */
  KET_OP_CSRSWAP = 7,     /* q = {c, a, b}                 (applyCsrSwap, :177)                  */
  KET_OP_UNITARY = 8,     /* q[0..nq-1], q[0] = MSB; 2^nq x 2^nq (applyUnitary, :240)           */
  KET_OP_BARRIER = 9,     /* no effect on the state                                               */
  KET_OP_MEASURE = 10,    /* q = {qubit, classical bit or -1 (not recorded)} (applyOps, circuit.ts:184-190) */
  KET_OP_RESET = 11,      /* q = {qubit}                   (circuit.ts:191-196)                  */
  KET_OP_IF = 12          /* q = {first classical bit, register size (<= 31), value, body length};
                             the body is the next `body length` ops, nested ifs included
                             (circuit.ts:197-199)                                                 */
} ket_op_kind;

#define KET_MAX_OP_QUBITS 10
#define KET_MAX_QUBITS 40

typedef struct ket_op {
  int32_t kind;                    /* ket_op_kind */
  int32_t nq;                      /* number of valid entries in q[] */
  int32_t q[KET_MAX_OP_QUBITS];
  int64_t mat;                     /* SINGLE/CONTROLLED/TWO/UNITARY: offset, in complex entries,
                                      of the row-major matrix in the caller's matrix buffer
                                      (interleaved re,im doubles); ignored otherwise */
} ket_op;

typedef struct ket_exec_opts {
  int32_t fusion;      /* -1 = automatic (default), 0 = one pass per gate, k > 0 = tile width cap (qubits) */
  int32_t prune;       /* 1 = reference accumulate() semantics: every computed amplitude with
                          |a|^2 < 1e-14 is flushed to zero (statevector.ts:19-27); 0 = plain dense */
  int32_t specialize;  /* register-tiled passes: 0 = automatic (default): kernels compiled for the
                          pass's program where one is ready (from earlier runs or ket_jit_compile),
                          the interpreter otherwise, compiling on background threads for states of
                          26+ qubits; 1 = compile what is
                          missing first, then use compiled kernels only; -1 = interpreter only.
                          Results are identical either way.  No counterpart in the reference. */
  int32_t reg_bits;    /* register bits of the compiled kernels' programs: 0 = automatic (default:
                          5 below 26 qubits, 4 from there on), 4 or 5 = that count at any size, so
                          that the programs large states run can be checked on small ones.  The
                          interpreter always uses 5.  No counterpart in the reference. */
  int32_t stage;       /* compiled kernels' tile loads: 1 = staged in shared memory by TMA copies
                          (one CTA per SM: two tile groups, each tile's copy issued while the
                          tile before it computes), -1 = loads
                          into registers (two CTAs per SM), 0 = automatic.  Results are identical
                          either way.  No counterpart in the reference. */
  int32_t reserved[3];
} ket_exec_opts;

/* NoiseParams (circuit.ts:213-221): depolarizing probability per single-qubit
 * gate, per two-qubit gate, and the readout flip probability. */
typedef struct ket_noise {
  double p1, p2, pmeas;
} ket_noise;

typedef struct ket_ctx ket_ctx;
typedef struct ket_state ket_state;

/* ---------------------------------------------------------------- context, memory */
KET_API const char* ket_last_error(void);
KET_API int ket_abi_version(void);
KET_API void ket_exec_opts_default(ket_exec_opts* opts);

/* One context per device; owns one CUDA stream and the scratch buffers. */
KET_API int ket_ctx_create(int device, ket_ctx** out);
KET_API int ket_ctx_destroy(ket_ctx* ctx);
/* Device memory currently held by the context's scratch pool (bytes). */
KET_API int ket_ctx_scratch_bytes(const ket_ctx* ctx, uint64_t* out);
/* Per-launch timing: with profiling on, every kernel the context launches is
 * bracketed by CUDA events on its stream; ket_ctx_profile_read waits for the
 * stream, returns (kind, milliseconds) per launch since the last read and
 * clears the list.  Kinds: 0 register-tiled fused pass, 1 small-state fused
 * pass, 2 single-gate pass, 3 read-out, 4 adjoint sweep, 5 batch.  No
 * counterpart in the reference (which only times whole calls, benchmark/run.mjs:16-35). */
KET_API int ket_ctx_profile(ket_ctx* ctx, int enable);
KET_API int ket_ctx_profile_read(ket_ctx* ctx, int* kinds, float* ms, size_t cap, size_t* count);
/* The context's CUDA stream (a cudaStream_t), so that a caller can order its
 * own work or record timing events against the engine's launches.  No
 * counterpart in the reference. */
KET_API int ket_ctx_stream(const ket_ctx* ctx, void** stream);
/* The device's FP64 fused-multiply-add rate (FMAs per second), measured by a
 * register-only kernel timed with CUDA events on the context's stream: the
 * FP64 roofline denominator of shared-memory-resident work (batched circuits,
 * small states).  No counterpart in the reference. */
KET_API int ket_measure_fp64(ket_ctx* ctx, double* fma_per_s);
/* Kernel launches made by the context so far. */
KET_API int ket_ctx_launch_count(const ket_ctx* ctx, uint64_t* count);
/* Bytes the context has copied host->device and device->host so far. */
KET_API int ket_ctx_io_bytes(const ket_ctx* ctx, uint64_t* h2d, uint64_t* d2h);
/* Host-side fault injection for tests: the after-th device allocation from now
 * on (0 = the next one) fails with KET_ERR_OOM; a negative value disables it.
 * No counterpart in the reference (which has no allocator). */
KET_API int ket_debug_fail_alloc(int after);
/* Test hook for the bounded waits of ket_batch_qaoa: drop_item >= 0 removes that
 * work item from the queue (tiles that depend on it then wait in vain) and
 * spin_limit sets how many polls a wait makes before it gives up and the call
 * returns KET_ERR_TIMEOUT (0 = the default, 2^24); drop_item = -1 disables.
 * No counterpart in the reference (which has no device waits). */
KET_API int ket_debug_batch_hook(int drop_item, uint32_t spin_limit);
/* Test hook for ket_adjoint_gradient's checkpoints: at most device_bytes of
 * device memory go to checkpoints of psi, the rest to pinned host memory
 * (a negative value: whatever free device memory allows, keeping 2 GiB
 * spare -- the default).  No counterpart in the reference. */
KET_API int ket_debug_adjoint_budget(int64_t device_bytes);
/* Test hook for the bounded waits of the staged pass kernels
 * (ket_exec_opts.stage = 1): tile >= 0 makes each such kernel skip the copies
 * of that tile, so the tile group's wait for it runs out (about
 * two seconds) and the call returns KET_ERR_TIMEOUT with the context still
 * usable; -1 disables.  No counterpart in the reference. */
KET_API int ket_debug_stage_drop(int64_t tile);

/* Dense state of 2^nqubits amplitudes, resident in device memory, set to |0..0>
 * (zero(n), statevector.ts:16).  precision: KET_C128 or KET_C64. */
KET_API int ket_state_alloc(ket_ctx* ctx, int nqubits, int precision, ket_state** out);
KET_API int ket_state_free(ket_state* st);
KET_API int ket_state_qubits(const ket_state* st, int* nqubits, int* precision);
/* |idx> (svFromBitstring, circuit.ts:136-140; the host reverses the q0-leftmost string). */
KET_API int ket_state_set_basis(ket_state* st, uint64_t idx);
/* Upload / download amplitudes [offset, offset+count) as interleaved FP64 (re, im). */
KET_API int ket_state_set_amplitudes(ket_state* st, uint64_t offset, uint64_t count, const double* re_im);
KET_API int ket_state_get_amplitudes(const ket_state* st, uint64_t offset, uint64_t count, double* re_im);
/* Copy src into dst (same size and precision). */
KET_API int ket_state_copy(ket_state* dst, const ket_state* src);

/* ---------------------------------------------------------------- circuit JSON */
/* A circuit loaded from ket's JSON (schema "ket": 1, the output of
 * Circuit.toJSON, circuit.ts:3768-3778), lowered to this ABI's op list. */
typedef struct ket_program ket_program;
/* Circuit.fromJSON (circuit.ts:3794-3806, opsFromJSON :532-580): parse the
 * text, rebuild every gate matrix from its meta name and parameters (:467-529),
 * inline named sub-circuits (flattenOps, :113-133) and pack measure / reset / if
 * for ket_run_shots, the registers of "cregs" taking consecutive classical bits
 * in the file's order.  KET_ERR_TYPE for malformed JSON, another schema
 * version, an unknown op kind or gate name, or unbound parameters (the
 * reference's TypeErrors). */
KET_API int ket_program_from_json(const char* text, size_t len, ket_program** out);
KET_API int ket_program_free(ket_program* p);
/* Qubits, ops, complex matrix entries, classical bits, registers, and whether
 * the op list holds measure / reset / if (then it runs with ket_run_shots). */
KET_API int ket_program_info(const ket_program* p, int* nqubits, size_t* nops, size_t* nmat, int* ncbits, int* nregs,
                             int* classical);
/* Copy out the op list and the matrices (2 * nmat doubles). */
KET_API int ket_program_ops(const ket_program* p, ket_op* ops, size_t ops_cap, double* mats, size_t mat_cap);
/* Register i: its name (NUL-terminated, truncated to cap bytes), first classical bit and size. */
KET_API int ket_program_creg(const ket_program* p, int i, char* name, size_t cap, int* first, int* size);

/* ---------------------------------------------------------------- running circuits */
/* simulatePure (circuit.ts:143-161): apply ops in order.  mats holds nmat complex
 * entries (2*nmat doubles).  Validation mirrors #checkOp (circuit.ts:1113-1146)
 * and happens before any launch: on error the state is unchanged. */
KET_API int ket_apply_ops(ket_state* st, const ket_op* ops, size_t nops, const double* mats, size_t nmat,
                  const ket_exec_opts* opts);

/* Planner statistics for an op list on an n-qubit state without launching
 * anything (no GPU needed): passes[0] = fused tile passes, passes[1] = single-
 * gate passes, passes[2] = gates absorbed.  Used by host-side tests. */
KET_API int ket_plan_stats(int nqubits, int precision, const ket_op* ops, size_t nops, const double* mats, size_t nmat,
                   const ket_exec_opts* opts, int64_t passes[3]);

/* Same, for the register-tiled passes: counts[t] = number of program ops of type t
 * (0 layout exchange, 1/2 2x2 on a register/lane bit, 3/4 X on a register/lane
 * bit, 5 register swap, 6 4x4, 7-10 diagonal forms, 11 merged phase fans and
 * phase polynomials), counts[12] / counts[13] =
 * 2x2 ops with a general / a real or Rx-like matrix, counts[14] = tiled passes,
 * counts[15] = other passes.  Programs use the register bits a run with these
 * options would (opts->reg_bits, else the automatic choice for nqubits).  No
 * counterpart in the reference. */
KET_API int ket_plan_program_stats(int nqubits, int precision, const ket_op* ops, size_t nops, const double* mats,
                                   size_t nmat, const ket_exec_opts* opts, int64_t counts[16]);

/* Run-time compiled pass kernels (ket_exec_opts.specialize).  ket_jit_wait
 * blocks until no compile is queued or running (KET_ERR_CUDA if one failed);
 * ket_jit_stats: out = {kernels known, compiled, failed, launches} and the
 * compile seconds summed over threads.  ket_jit_compile plans an op list as
 * ket_apply_ops would for an nqubits state and compiles, on all host cores,
 * the kernel of every register-tiled pass that is not compiled yet (no GPU
 * needed); *kernels = the number of distinct kernels the plan uses, log = a
 * failed compile's log (logcap bytes).  No counterpart in the reference. */
KET_API int ket_jit_wait(void);
/* Drop queued background compiles and wait for the running ones (each takes
 * about a second).  A host calls it before exiting: a compile still running
 * while the process tears down NVRTC would crash the exit.  The Python
 * binding registers it with atexit; the N-API addon with
 * napi_add_env_cleanup_hook. */
KET_API int ket_jit_shutdown(void);
KET_API int ket_jit_stats(int64_t out[4], double* compile_seconds);
KET_API int ket_jit_compile(int nqubits, int precision, const ket_op* ops, size_t nops, const double* mats,
                            size_t nmat, const ket_exec_opts* opts, int64_t* kernels, char* log, size_t logcap);

/* ---------------------------------------------------------------- read-outs */
/* amplitude(): out[2i], out[2i+1] = re, im of amplitude idx[i] (circuit.ts:1491-1495). */
KET_API int ket_amplitudes(const ket_state* st, const uint64_t* idx, size_t k, double* out_re_im);
/* probabilities() as a dense array: out[i] = |a_i|^2 if > threshold else 0
 * (statevector.ts:273-280 with threshold 1e-14). */
KET_API int ket_probs_dense(const ket_state* st, double threshold, double* out);
/* exactProbs() (circuit.ts:3700-3711): entries with p > threshold in ascending index
 * order.  Writes min(count, cap) entries; *count = total number of such entries. */
KET_API int ket_probs_sparse(const ket_state* st, double threshold, uint64_t* idx, double* p, uint64_t cap,
                     uint64_t* count);
/* marginals() (circuit.ts:1508-1518): out[q] = P(qubit q = 1), q = 0..n-1. */
KET_API int ket_marginals(const ket_state* st, double* out);
/* marginals() for callers that cannot allocate device memory (code inside
 * another framework's memory pool or allocator hooks, or that only lends
 * buffers it already owns).  amp: the caller's device array of 2^nqubits
 * amplitudes (precision KET_C128 or KET_C64); out: the caller's device array of
 * nqubits doubles, out[q] = P(qubit q = 1).  The work is queued on `stream` (a
 * cudaStream_t, NULL = the default stream) and the call returns without
 * waiting.  The reduction scratch is a fixed device array of
 * KET_NOALLOC_SCRATCH_BYTES held by every GPU that loads the library until the
 * process exits; the call allocates nothing and rejects sizes whose scratch
 * would exceed it.  The first call on a device looks the array up
 * (cudaGetSymbolAddress) and should come before any stream capture.  All calls
 * share the array: calls that overlap on the GPU race and give wrong results.
 * amp and out must be device (or managed) memory of the current device, else
 * KET_ERR_TYPE.  The array's address is kept per device for the life of the
 * process, so the call must not be used on a device after cudaDeviceReset.
 * No counterpart in the reference. */
#define KET_NOALLOC_SCRATCH_BYTES (2048u * 40u * 8u)
KET_API int ket_marginals_noalloc(const void* amp, int nqubits, int precision, double* out, void* stream);
/* Joint distribution of m qubits: out[j] = P(bit k of j = qubit qubits[k], for all k), 2^m bins (1 <= m <= 12). */
KET_API int ket_marginal_dist(const ket_state* st, const int* qubits, int m, double* out);
/* Compare two states of the same size (any precisions, same context):
 * overlap = <a|b> (re, im) and max_abs_diff = max_i |a_i - b_i|, accumulated in
 * FP64.  States the fidelity and amplitude error of a complex64 state against a
 * complex128 one.  No counterpart in the reference. */
KET_API int ket_state_compare(const ket_state* a, const ket_state* b, double* overlap_re_im, double* max_abs_diff);
/* Sum of |a|^2 (FP64 accumulation). */
KET_API int ket_norm2(const ket_state* st, double* out);
/* run() pure fast path sampler (circuit.ts:3424-3453): r[s] are the caller's
 * uniform draws (makePrng, circuit.ts:813-819), each in [0, 1] (KET_ERR_RANGE
 * otherwise); out_idx[s] = the first index, in ascending order over entries with
 * p > threshold, whose running FP64 sum is >= r[s] (the last such entry's running sum
 * is taken as 1.0).  The running sum is the reference's, rounded after every
 * addition in ascending index order, bit for bit at every state size. */
KET_API int ket_sample(const ket_state* st, const double* r, size_t shots, double threshold, uint64_t* out_idx);
/* circuitMatrix() (circuit.ts:1462-1485): the 2^n x 2^n matrix of ops on
 * nqubits <= 12 (KET_ERR_RANGE above, as the reference), out[row * 2^n + col]
 * as interleaved (re, im), rows and columns indexed with q0 as the MOST
 * significant bit (the standard convention the reference uses here).  Column
 * col is the state the ops make from |flip(col)>, with the reference's
 * per-gate pruning.  Allocates a 2n-qubit device state for the call. */
KET_API int ket_circuit_matrix(ket_ctx* ctx, int nqubits, const ket_op* ops, size_t nops, const double* mats,
                               size_t nmat, const ket_exec_opts* opts, double* out);
/* blochAngles(q) (circuit.ts:4102-4129): out = {rho00, rho11, Re rho01,
 * Im rho01, theta, phi} of qubit q's reduced density matrix, with
 * theta = acos(clamp(rho00 - rho11)) and phi = atan2(-2 Im rho01, 2 Re rho01). */
KET_API int ket_bloch(const ket_state* st, int q, double* out);
/* runDM (density.ts:475-588, Circuit.dm() circuit.ts:4562-4579): the exact
 * density matrix of ops on n qubits from |0..0><0..0|, with per-gate
 * depolarizing noise p1 (after single-qubit gates) and p2 (after cnot / swap /
 * two / controlled); p <= 0 adds none.  rho is a state of 2n qubits holding
 * rho[row][col] at index (row << n) | col; each op runs as U rho U^dagger with
 * the reference's pruning of every output entry below |v|^2 = 1e-14.
 * Unitary ops of more than 5 qubits: KET_ERR_UNSUPPORTED.  Read the result
 * with ket_amplitudes / ket_state_get_amplitudes (entries), ket_norm2
 * (purity, density.ts:314-318), ket_dm_probs and ket_dm_bloch. */
KET_API int ket_dm_run(ket_state* rho, const ket_op* ops, size_t nops, const double* mats, size_t nmat, double p1,
                       double p2);
/* The diagonal of rho: out[r] = Re rho[r][r] (DensityMatrix.probabilities,
 * density.ts:299-307, before its p > 1e-14 filter), 2^n values. */
KET_API int ket_dm_probs(const ket_state* rho, double* out);
/* DensityMatrix.blochAngles(q) (density.ts:356-372): out = {theta, phi}. */
KET_API int ket_dm_bloch(const ket_state* rho, int q, double* out);
/* run()'s per-shot path (circuit.ts:3455-3481 over applyOps, :169-207): one
 * trajectory per shot from |init>, using st as the device workspace (its
 * qubit count and precision; its contents are overwritten).  ops may hold
 * measure / reset / if (KET_OP_MEASURE...).  noise (NULL = none) adds the
 * depolarizing Paulis of dep1 / dep2 (:289-304) after single-qubit gates and
 * after cnot / controlled / swap / two, and the readout flips.  All shots
 * share one xorshift32 stream whose state is *prng_state (makePrng,
 * :813-819; 0 reads as 1), drawn in the reference's order; on return it holds
 * the state after the last draw.  ncbits = classical bits of all registers,
 * numbered consecutively.  Outputs per shot s: out_idx[s] = the sampled basis
 * index after readout flips (sampleSV, :75-83), out_bits[s * ncbits + b] =
 * classical bit b at the end of the shot.  P(q=1) is summed in a fixed device
 * order where the reference sums in its Map's insertion order: the two agree
 * up to rounding. */
KET_API int ket_run_shots(ket_state* st, const ket_op* ops, size_t nops, const double* mats, size_t nmat,
                          const ket_noise* noise, uint64_t init, size_t shots, uint32_t* prng_state, int ncbits,
                          uint64_t* out_idx, uint8_t* out_bits);
/* Test hook for ket_run_shots: 0 = automatic (states of up to 12 qubits c128
 * / 13 c64 whose shots draw a fixed number of times run as batched
 * trajectories, one CTA per shot with the state in shared memory; others
 * run one trajectory at a time through the fused engine), 1 = always one at
 * a time, 2 = batched only (KET_ERR_UNSUPPORTED where it does not apply).
 * No counterpart in the reference. */
KET_API int ket_debug_pershot_path(int mode);
/* Circuit.expectation(pauli) (circuit.ts:3728-3753): pauli[q] in "IXYZ" acts on qubit q. */
KET_API int ket_expect_pauli(const ket_state* st, const char* pauli, double* out);
/* vqe() energy (algorithms.ts:301-336): sum_t coeffs[t] <P_t>.  ops holds nterms
 * strings of n characters back to back; ops[t*n + 0] acts on qubit n-1 (the
 * PauliTerm convention, algorithms.ts:283-285).  Terms with |coeff| < 1e-15 are
 * skipped and all-identity terms add coeff, as the reference does. */
KET_API int ket_expect_pauli_sum(const ket_state* st, int nterms, const double* coeffs, const char* ops, double* out);

/* ---------------------------------------------------------------- differentiation */
/* Parametric gates of a circuit template (the 'parametric' ops of circuit.ts:39-43
 * after bind(), resolveParametric circuit.ts:1047-1073).  The angle fed to the gate
 * is scale * params[param] + shift. */
typedef enum ket_param_gate {
  KET_PG_RX = 0, KET_PG_RY = 1, KET_PG_RZ = 2, KET_PG_U1 = 3,     /* single-qubit (rz also vz; u1 also p) */
  KET_PG_GPI = 4, KET_PG_GPI2 = 5,
  KET_PG_CRX = 6, KET_PG_CRY = 7, KET_PG_CRZ = 8, KET_PG_CU1 = 9, /* controlled: q = {c, t} */
  KET_PG_XX = 10, KET_PG_YY = 11, KET_PG_ZZ = 12, KET_PG_XY = 13  /* two-qubit: q = {a, b} */
} ket_param_gate;

typedef struct ket_param_binding {
  int32_t op;        /* index into the template's op list; that op's matrix is replaced */
  int32_t gate;      /* ket_param_gate */
  int32_t param;     /* parameter index */
  int32_t reserved;
  double scale;      /* angle = scale * params[param] + shift */
  double shift;
} ket_param_binding;

/* Adjoint gradient of E(theta) = <psi(theta)|H|psi(theta)>, psi(theta) = U(theta)|init>,
 * for `batch` parameter vectors (params[b*nparams + k]).  Replaces gradient() by parameter
 * shift (algorithms.ts:536-547), which costs 2*nparams energy evaluations.  The template
 * ops carry placeholder matrices for bound ops; H is a PauliTerm list (see
 * ket_expect_pauli_sum).  energy[b] and grad[b*nparams + k] are written.
 * checkpoint_every: 0 = automatic (8 sqrt(#ops)), -1 = none; the forward state is
 * stored every that many ops and restored during the reverse sweep, in device
 * memory while free memory holds it and in pinned host memory beyond that.  The
 * vectors of a batch are queued without host waits, and a batch of 8 or more
 * runs its passes on kernels compiled for their programs. */
KET_API int ket_adjoint_gradient(ket_ctx* ctx, int nqubits, uint64_t init, const ket_op* ops, size_t nops,
                         const double* mats, size_t nmat, const ket_param_binding* binds, size_t nbinds,
                         const double* params, int nparams, int batch, int nterms, const double* coeffs,
                         const char* pauli_ops, int checkpoint_every, double* energy, double* grad);

/* Parameter-shift gradient on the same engine, the reference's algorithm
 * (gradient(), algorithms.ts:536-547): 2*nparams + 1 full simulations per
 * parameter vector, grad_k = (E(theta + pi/2 e_k) - E(theta - pi/2 e_k)) / 2.
 * prune: 1 = the reference's per-gate pruning, 0 = plain dense.  Same arguments
 * as ket_adjoint_gradient otherwise. */
KET_API int ket_shift_gradient(ket_ctx* ctx, int nqubits, uint64_t init, const ket_op* ops, size_t nops,
                               const double* mats, size_t nmat, const ket_param_binding* binds, size_t nbinds,
                               const double* params, int nparams, int batch, int nterms, const double* coeffs,
                               const char* pauli_ops, int prune, double* energy, double* grad);

/* ---------------------------------------------------------------- batching */
/* QAOA MaxCut batch: instance i has n[i] qubits, ne[i] edges at edges[2*eoff[i] ...],
 * p layers with gamma[i*p + l], beta[i*p + l].  Circuit: H on all qubits, then per layer
 * exp(-i gamma Z_u Z_v) on every edge and Rx(2 beta) on every qubit.  out[i] = <C> =
 * sum_edges (1 - <Z_u Z_v>)/2 in FP64.  This equals vqe(qaoa(n, E, -2*gamma, beta),
 * maxCutHamiltonian(n, E)) of algorithms.ts:231-276.  All instances run in one
 * persistent launch (captured in a CUDA graph and replayed when use_graph = 1). */
/* Launch shape of ket_batch_qaoa on this context: block_threads in {128, 256,
 * 512} threads per CTA and tile_bits in {11, 12} (instances up to tile_bits
 * qubits run whole in shared memory; wider ones, up to 2 * tile_bits qubits,
 * as tiled passes).  0 selects the default (256, 12).  The autotuner in
 * ket_b200/autotune.py picks them per workload.  No counterpart in the reference. */
KET_API int ket_batch_config(ket_ctx* ctx, int block_threads, int tile_bits);
KET_API int ket_batch_qaoa(ket_ctx* ctx, int ninst, const int* n, const int* ne, const int64_t* eoff, const int* edges,
                   int p, const double* gamma, const double* beta, int use_graph, double* out);

/* A circuit template of ket_batch_vqe: ops[op_first .. op_first + nops) on
 * nqubits qubits (1..13), its parametric ops bound by binds[bind_first ..
 * bind_first + nbinds) (op indices relative to op_first, placeholder matrices
 * in the op list as for ket_adjoint_gradient), and its Hamiltonian: nterms
 * PauliTerms with coefficients coeffs[term_first ..] and strings of nqubits
 * characters each at pauli[pauli_first ..] (ops[0] acts on qubit n-1). */
typedef struct ket_batch_template {
  int32_t nqubits, nops, nbinds, nterms;
  int64_t op_first, bind_first, term_first, pauli_first;
} ket_batch_template;

/* vqe() (algorithms.ts:301-336) over a batch of parameterised circuits: instance
 * i runs template inst_template[i] at parameters theta[i*nparams ..] from
 * |0...0> with the reference's per-gate pruning and returns
 * energy[i] = sum_t coeff_t <psi_i|P_t|psi_i>, as a parameter sweep of
 * vqe(ansatz(params), H) would, one call per instance.  Templates may differ in
 * qubit count, gates and Hamiltonian.  All instances run in one persistent
 * launch (one CTA per instance with its state in shared memory, widest first);
 * with use_graph = 1 the launch is captured in a CUDA graph that later calls of
 * the same shape replay.  Ops: single, controlled, two, unitary of 1-2 qubits,
 * cnot, swap, toffoli, cswap, csrswap, barrier. */
KET_API int ket_batch_vqe(ket_ctx* ctx, int ntemplates, const ket_batch_template* templates, const ket_op* ops,
                          const double* mats, size_t nmat, const ket_param_binding* binds, const double* coeffs,
                          const char* pauli, int ninst, const int* inst_template, const double* theta, int nparams,
                          int use_graph, double* energy);

#ifdef __cplusplus
}
#endif

#endif /* KET_SV_H */
