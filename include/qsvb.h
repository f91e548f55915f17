/* qsvb.h — C ABI of the B200 statevector engine (libqsvb.so).
 *
 * This is the drop-in boundary for qsv's `Backend<R>` trait
 * (crates/qsv-core/src/backend/mod.rs:31-74). A thin host shim (Rust `impl Backend<f32>` /
 * `impl Backend<f64>`, or the Python mirror in rustatevec_b200/backend.py) forwards each trait
 * method to one call below and turns a non-zero status into the trait's panic.
 *
 * Conventions
 *  - Every entry point returns an `int` status: QSVB_OK (0) or a negative QSVB_E_* code. No C++
 *    exception crosses this boundary. qsvb_last_error() returns the message of the calling
 *    thread's most recent failure.
 *  - States are opaque handles owned by the caller (alloc/free). Pointers passed in are borrowed
 *    for the duration of the call.
 *  - Work is queued on the context's CUDA stream. Calls that return data to the host
 *    (download, probabilities, amplitude, reductions) synchronize that stream first.
 *  - Gate convention (crates/qsv-core/src/gate.rs:8-13): bit j of a gate's row/column index is
 *    state bit qubits[j]; controlled gates list the control first.
 *  - Matrices are row-major 2^m x 2^m, complex as interleaved (re, im) FP64. A complex64 state
 *    rounds them to f32 on use (the rounding of Cplx::from_f64); fused gates are composed in FP64.
 *  - A context is not thread-safe: use one context per host thread.
 */
#ifndef QSVB_H
#define QSVB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QSVB_OK 0
#define QSVB_E_INVALID -1     /* bad argument: qubit out of range, repeated qubit, arity, null */
#define QSVB_E_CUDA -2        /* a CUDA runtime/driver call failed */
#define QSVB_E_OOM -3         /* device memory exhausted */
#define QSVB_E_UNSUPPORTED -4 /* valid request this build cannot serve */
#define QSVB_E_TIMEOUT -5     /* a bounded device-side wait ran out (persistent runner) */

#define QSVB_MAX_GATE_QUBITS 6
#define QSVB_MAX_QUBITS 34

typedef enum qsvb_dtype { QSVB_C64 = 0, QSVB_C128 = 1 } qsvb_dtype;

typedef struct qsvb_ctx qsvb_ctx;
typedef struct qsvb_state qsvb_state;
typedef struct qsvb_plan qsvb_plan;

/* One gate application (crates/qsv-core/src/circuit.rs:13-16 GateOp). */
typedef struct qsvb_gate {
  uint32_t n_qubits;                       /* m, 1..6 */
  uint32_t qubits[QSVB_MAX_GATE_QUBITS];   /* gate order; entries >= m are ignored */
  const double* matrix;                    /* 2^m x 2^m, row-major, interleaved (re, im) */
} qsvb_gate;

/* A circuit (crates/qsv-core/src/circuit.rs:31-34). */
typedef struct qsvb_circuit {
  uint32_t n_qubits;
  size_t n_gates;
  const qsvb_gate* gates;
} qsvb_circuit;

/* Planner choices for qsvb_execute / qsvb_plan_create. */
typedef enum qsvb_planner {
  QSVB_PLAN_AS_GIVEN = 0, /* one sweep per gate, in order (the trait's default execute loop) */
  QSVB_PLAN_GREEDY = 1,   /* qsv fuse semantics (fusion.rs:39-77), composition in FP64 */
  QSVB_PLAN_WINDOW = 2,   /* commutation-aware windows: gates on disjoint qubits reorder */
  QSVB_PLAN_LEARNED = 3,  /* cost-model planner (MLP cost model; greedy fallback); also weighs
                             tile passes against fused sweeps */
  QSVB_PLAN_TILE = 4,     /* tile passes: the 1- and 2-qubit gates acting inside a set of up to
                             12 qubits (11 for complex128) that commute past the gates left for
                             later, applied on shared-memory tiles in one read and one write of
                             the state; diagonal runs become phase sweeps, wider gates fused sweeps */
  QSVB_PLAN_CHAIN = 5     /* tensor-core chain passes (complex64, n >= 12): each pass takes a set of
                             12 qubits, applies up to chain_max_matrices fused 6-qubit matrices of
                             the gates inside it on tcgen05 in one read and one write of the state,
                             and relabels which qubits sit on the state's low bits for the next
                             pass; permutation passes put every qubit back on its own bit at the end.
                             Other states (complex128, n < 12, CUDA-core engine) plan as WINDOW. */
} qsvb_planner;

typedef enum qsvb_engine {
  QSVB_ENGINE_AUTO = 0,        /* tensor cores for k>=5 complex64 sweeps, CUDA cores otherwise */
  QSVB_ENGINE_CUDA_CORE = 1,   /* all dense sweeps on CUDA cores (FP32 / FP64) */
  QSVB_ENGINE_TENSOR_CORE = 2  /* dense complex64 sweeps with k>=4 on tcgen05 (BF16 hi/lo) */
} qsvb_engine;

typedef struct qsvb_plan_opts {
  uint32_t planner;          /* qsvb_planner */
  uint32_t max_fused_qubits; /* fusion width cap, 1..6 (ignored by AS_GIVEN) */
  uint32_t engine;           /* qsvb_engine */
  uint32_t use_graph;        /* reusable plans: capture the sweep sequence in a CUDA graph */
  uint32_t chain_max_matrices; /* QSVB_PLAN_CHAIN: matrices per pass, 1..3 (0: chosen by cost) */
  uint32_t reserved[3];
} qsvb_plan_opts;

/* What a plan does, for reports and rooflines. */
typedef struct qsvb_plan_stats {
  uint64_t n_gates_in;        /* gates in the input circuit */
  uint64_t n_sweeps;          /* kernel sweeps launched per run */
  uint64_t n_sweeps_by_kind[10]; /* 1q, ctrl1q, diag, phase, dense CUDA-core, dense TC, tile pass,
                                   other, tensor-core chain pass, tile permutation */
  double algorithmic_bytes;   /* sum over sweeps of 2 * (amplitudes the sweep may change) * bytes/amp */
  double full_sweep_bytes;    /* sum over sweeps of 2 * 2^n * bytes/amp */
  double flops;               /* complex-MAC flops of the dense sweeps (8 * 2^k per amplitude) */
  double predicted_seconds;   /* planner's cost-model estimate (0 where nothing is predicted) */
  double measured_seconds;    /* device seconds measured by the call itself (qsvb_execute_batch*,
                                 qsvb_batch_run); 0 where the call measures nothing */
} qsvb_plan_stats;

/* ---------------------------------------------------------------- lifecycle */
/* Backend construction (crates/qsv-cuda/src/lib.rs:57-77 CudaBackend::new). */
int qsvb_create(int device_ordinal, qsvb_ctx** out);
int qsvb_destroy(qsvb_ctx* ctx);
const char* qsvb_last_error(void);
int qsvb_synchronize(qsvb_ctx* ctx);
/* Library version string, e.g. "qsvb 0.1 sm_100a". */
const char* qsvb_version(void);
/* The context's CUDA stream (a cudaStream_t), so callers can order their own work and record
 * CUDA events against the engine's queue. */
int qsvb_stream(qsvb_ctx* ctx, void** stream_out);

/* Backend::alloc (mod.rs:36; lib.rs:100-107). Contents unspecified until init/upload. */
int qsvb_state_alloc(qsvb_ctx* ctx, uint32_t n_qubits, int dtype, qsvb_state** out);
int qsvb_state_free(qsvb_ctx* ctx, qsvb_state* st);
/* Shape of a state and its device SoA pointers (re[2^n], im[2^n]). */
int qsvb_state_info(const qsvb_state* st, uint32_t* n_qubits, int* dtype, void** d_re, void** d_im);

/* ---------------------------------------------------------------- state preparation */
/* Backend::init_basis (mod.rs:39; lib.rs:109-119). */
int qsvb_init_basis(qsvb_ctx* ctx, qsvb_state* st, uint64_t basis);
/* Arbitrary-state upload from host SoA arrays in the state's precision (no trait counterpart). */
int qsvb_upload(qsvb_ctx* ctx, qsvb_state* st, const void* re, const void* im);
/* Seeded i.i.d. complex Gaussian amplitudes normalised in FP64 (no trait counterpart). */
int qsvb_init_gaussian(qsvb_ctx* ctx, qsvb_state* st, uint64_t seed);

/* ---------------------------------------------------------------- gate application */
/* Backend::apply (mod.rs:42; lib.rs:121-200): one gate, dispatched to a fast path. */
int qsvb_apply(qsvb_ctx* ctx, qsvb_state* st, const double* matrix, const uint32_t* qubits,
               uint32_t n_qubits);
/* Backend::execute (mod.rs:66-73) on an initialised state: plans, uploads matrices once, and
 * launches every sweep directly (use_graph applies to reusable plans: a graph instantiated for a
 * single run would only hold back the first kernel). opts may be NULL (greedy, k=4, auto
 * engine). stats may be NULL. */
int qsvb_execute(qsvb_ctx* ctx, qsvb_state* st, const qsvb_circuit* circuit,
                 const qsvb_plan_opts* opts, qsvb_plan_stats* stats);

/* Reusable plans: plan once, run many times (the graph is instantiated on first run). */
int qsvb_plan_create(qsvb_ctx* ctx, const qsvb_circuit* circuit, int dtype,
                     const qsvb_plan_opts* opts, qsvb_plan** out);
int qsvb_plan_run(qsvb_ctx* ctx, qsvb_plan* plan, qsvb_state* st);
int qsvb_plan_stats_get(const qsvb_plan* plan, qsvb_plan_stats* out);
int qsvb_plan_free(qsvb_ctx* ctx, qsvb_plan* plan);

/* One sweep of a plan, as the planner and the cost model see it. */
typedef struct qsvb_sweep_info {
  uint32_t kind;                  /* 0 1q, 1 ctrl1q, 2 diag, 3 phase, 4 dense CUDA-core, 5 dense TC,
                                     6 tile pass, 8 tensor-core chain pass, 9 tile permutation */
  uint32_t n_qubits;              /* matrix qubits (dense/diag); matrices of a chain pass */
  uint32_t qubits[QSVB_MAX_GATE_QUBITS]; /* chain / permutation passes: the tile's state bits
                                            above bit 5 */
  uint32_t target;                /* butterflies */
  uint32_t n_ctrl;                /* controls (ctrl1q) or skipped identity halves (diag) */
  uint32_t ctrl[QSVB_MAX_GATE_QUBITS];
  uint32_t n_terms;               /* phase polynomial terms */
  uint64_t n_gates;               /* input gates this sweep covers */
  double algorithmic_bytes;       /* 2 * (amplitudes it may change) * bytes per amplitude */
  double flops;                   /* 8 * 2^k per amplitude for dense sweeps */
  float features[16];             /* cost-model input vector */
} qsvb_sweep_info;
int qsvb_plan_sweep_info(const qsvb_plan* plan, size_t index, qsvb_sweep_info* out);
/* Device time of each sweep of `plan` on `st`: CUDA events around `reps` back-to-back launches of
 * each sweep; out_seconds[i] = mean seconds per launch of sweep i. The state is overwritten. */
int qsvb_plan_profile(qsvb_ctx* ctx, qsvb_plan* plan, qsvb_state* st, int reps, double* out_seconds);
/* Fused gate list a planner produces (crates/qsv-core/src/fusion.rs:39 fuse). Call with
 * out_gates == NULL to get the count in *n_out; matrices are written to out_mats (FP64
 * interleaved) with out_gates[i].matrix pointing into it. Needs no device. */
int qsvb_fuse(const qsvb_circuit* circuit, const qsvb_plan_opts* opts, qsvb_gate* out_gates,
              size_t* n_out, double* out_mats, size_t out_mats_cap);

/* Plans a circuit on the host without a device (no allocation, no upload): the statistics the
 * plan would report (sweeps by kind, algorithmic bytes, flops, predicted seconds), e.g. to compare
 * planners or check a plan before a 137 GB state exists. No trait counterpart. */
int qsvb_plan_dry_run(const qsvb_circuit* circuit, int dtype, const qsvb_plan_opts* opts,
                      qsvb_plan_stats* stats);

/* ---------------------------------------------------------------- read-out */
/* Every read-out call below waits for the context's queued work and reports a failure that work
 * flagged on the device (a bounded wait that ran out: QSVB_E_TIMEOUT; a failed range check of the
 * bounds-checked build: QSVB_E_CUDA), as qsvb_synchronize does; the state's contents are then
 * invalid. */
/* Backend::download (mod.rs:62; lib.rs:218-227): SoA copy into host buffers of the state's
 * precision. */
int qsvb_download(qsvb_ctx* ctx, const qsvb_state* st, void* re, void* im);
/* Backend::amplitude (mod.rs:45): one element (not the whole state as lib.rs:202-205 does). */
int qsvb_amplitude(qsvb_ctx* ctx, const qsvb_state* st, uint64_t index, double out[2]);
/* Backend::probabilities (mod.rs:48; lib.rs:207-216 k_abs2). |psi_i|^2 computed in FP64;
 * written to host `out` as f64 (out_dtype QSVB_C128) or rounded to f32 (QSVB_C64). */
int qsvb_probabilities(qsvb_ctx* ctx, const qsvb_state* st, void* out, int out_dtype);
/* Backend::expectation_z (mod.rs:57-59; sample.rs:177-200), FP64 on device. */
int qsvb_expectation_z(qsvb_ctx* ctx, const qsvb_state* st, uint64_t mask, double* out);
/* Backend::sample overridden on the device (mod.rs:52-54: "a device backend overrides this"),
 * drawing as cdf_sample does (crates/qsv-core/src/sample.rs:163-172): shot k returns the first
 * outcome i whose FP64 cumulative probability is >= u_k * total, u_k the k-th unit() value of
 * SplitMix64(seed) (crates/qsv-core/src/circuits.rs:22-46), i.e. seed = the caller's rng state
 * before the call, which then advances by `shots` draws. Probabilities are |amp|^2 rounded in the
 * state's precision, as Backend::probabilities computes them; the FP64 prefix sums run in another
 * order than the reference's, so a draw can differ only where u_k * total lies within rounding of
 * a cumulative value. No probability download. shots <= 2^30. */
int qsvb_sample(qsvb_ctx* ctx, const qsvb_state* st, uint64_t shots, uint64_t seed, uint64_t* out);
/* StateVector::norm_sqr (crates/qsv-core/src/state/mod.rs:112-118), FP64 on device. */
int qsvb_norm_sqr(qsvb_ctx* ctx, const qsvb_state* st, double* out);
/* <a|b> in FP64 (no trait counterpart). a and b may differ in precision (complex64 vs complex128),
 * which is how a complex64 run is scored against its FP64 twin. */
int qsvb_inner_product(qsvb_ctx* ctx, const qsvb_state* a, const qsvb_state* b, double out[2]);
/* <Z_mask> like qsvb_expectation_z, for callers that cannot allocate device memory: it takes the
 * caller's own device SoA buffers (re[2^n], im[2^n] in the precision `dtype`), a CUDA stream
 * (NULL = default stream) and a host `out`, needs no context, and calls no cudaMalloc / cudaFree.
 * Its reduction scratch is a fixed 16.4 KB __device__ array inside the library (held on every GPU
 * that loads it until exit; partial sums of at most 1024 CTAs; n_qubits up to 34, larger or
 * malformed requests return QSVB_E_INVALID). d_re and d_im must be device or managed memory of
 * the current device and 16-byte aligned; host pointers, another device's memory and misaligned
 * offsets return QSVB_E_INVALID before any launch. All calls share that array, so calls whose
 * kernels overlap on the GPU race; the first call on a device (and the first after a
 * cudaDeviceReset, which invalidates the array's address) sets the array up and must come before
 * any stream capture. No counterpart in the reference: it exists for hosts that run under a fixed
 * device-memory budget or own every device allocation themselves. Waits for its result. */
int qsvb_expectation_z_noalloc(const void* d_re, const void* d_im, uint32_t n_qubits, int dtype, uint64_t mask,
                               void* stream, double* out);
/* |<a|b>|^2 in FP64 (no trait counterpart). */
int qsvb_fidelity(qsvb_ctx* ctx, const qsvb_state* a, const qsvb_state* b, double* out);

/* ---------------------------------------------------------------- autotuner and learned cost model
 * (no trait counterpart: they replace the fixed max-k rule of fusion.rs:26-36 with a planner that
 * picks fusion width, strategy and kernel engine from predicted sweep times). */
/* Times candidate sweeps (every kind, k = 1..6, CUDA-core and tensor-core engines, several qubit
 * placements) on an n-qubit state (12 <= n <= 32): features[i*16..] is the cost-model input of
 * candidate i, seconds[i] its mean device time over `reps` launches, kinds[i] its sweep kind.
 * Call with features == NULL to get the candidate count in *count. */
int qsvb_autotune(qsvb_ctx* ctx, uint32_t n_qubits, int dtype, int reps, uint64_t seed, float* features,
                  double* seconds, uint32_t* kinds, size_t cap, size_t* count);
/* Trains the MLP cost model (16 -> hidden -> hidden -> 1, ReLU, predicts log2 seconds) on the
 * GPU with full-batch Adam and installs it for the learned planner. */
int qsvb_costmodel_train(qsvb_ctx* ctx, const float* features, const float* log2_seconds, size_t n,
                         uint32_t hidden, uint32_t epochs, float lr, uint64_t seed, float* final_loss);
/* One forward + backward pass on the GPU for given flat parameters (see mlp.cu for the layout) on
 * already-normalised inputs: mean-squared-error loss and its gradient (gradient checks). */
int qsvb_costmodel_forward_backward(qsvb_ctx* ctx, const float* params, uint32_t hidden, const float* x,
                                    const float* target, size_t n, float* loss, float* grad);
/* Installed model as a flat float image (call with out == NULL for its length); set installs an
 * image (NULL / 0 uninstalls: the planner falls back to its roofline model). */
int qsvb_costmodel_get(float* out, size_t cap, size_t* needed);
int qsvb_costmodel_set(const float* image, size_t len);
/* Host forward of the installed model: log2 seconds for each 16-float feature row. */
int qsvb_costmodel_predict(const float* features, size_t n, float* out_log2_seconds);

/* ---------------------------------------------------------------- batched circuits */
/* Many small independent circuits (each n <= 30, gates of 1 or 2 qubits) in one persistent
 * kernel. For circuit i the engine writes <Z_0> to z0_out[i] (when z0_out != NULL) and, when
 * probs_out != NULL, its 2^n_i FP64 probabilities at probs_out + probs_offset[i] (host memory),
 * or packed in circuit order when probs_offset == NULL. Each circuit starts from |0..0>.
 * stats (optional): n_sweeps = passes over shared-memory tiles, n_sweeps_by_kind[0] = register
 * phases, algorithmic_bytes = HBM bytes of those passes plus the probabilities, flops = gate
 * arithmetic, measured_seconds = measured device seconds of the batched kernels. Replaces a host
 * loop of Backend::execute over the circuits (crates/qsv-core/src/backend/mod.rs:66-73) followed
 * by expectation_z (crates/qsv-core/src/sample.rs:177-200). */
int qsvb_execute_batch(qsvb_ctx* ctx, const qsvb_circuit* circuits, size_t n_circuits, int dtype,
                       double* z0_out, double* probs_out, const uint64_t* probs_offset,
                       qsvb_plan_stats* stats);
/* A reusable batch: the plan (passes over HBM, register phases, work queue), its device buffers
 * and one CUDA graph with the per-run device work, built once; each run replays the graph and
 * copies <Z_0> (and, when asked, the probabilities) to the host. local_qubits / register_qubits
 * as in qsvb_execute_batch_ex. No trait counterpart. */
typedef struct qsvb_batch qsvb_batch;
int qsvb_batch_create(qsvb_ctx* ctx, const qsvb_circuit* circuits, size_t n_circuits, int dtype,
                      uint32_t local_qubits, uint32_t register_qubits, qsvb_batch** out);
int qsvb_batch_run(qsvb_ctx* ctx, qsvb_batch* batch, double* z0_out, double* probs_out,
                   const uint64_t* probs_offset, qsvb_plan_stats* stats);
/* Failure detection of the batched runner (no trait counterpart): a tile of pass p waits for
 * every tile of pass p-1 of its circuit; each such wait may take at most `cycles` clock64 cycles
 * (0 restores the default, 2^32, about 2 s; at most 2^40). A wait that runs out fails the run:
 * every block abandons its remaining work, and qsvb_batch_run returns QSVB_E_TIMEOUT with the
 * context still usable. */
int qsvb_batch_set_wait_budget(qsvb_ctx* ctx, qsvb_batch* batch, uint64_t cycles);
int qsvb_batch_free(qsvb_ctx* ctx, qsvb_batch* batch);
/* Times each tile shape (local qubits from two below the limit up to it, both register widths)
 * on this batch; writes the fastest to *best_local / *best_register and, when seconds != NULL,
 * the device seconds of each candidate (local-major order, at most cap; *count = number of
 * candidates). */
int qsvb_batch_autotune(qsvb_ctx* ctx, const qsvb_circuit* circuits, size_t n_circuits, int dtype,
                        uint32_t* best_local, uint32_t* best_register, double* seconds, size_t cap,
                        size_t* count);
/* Same as qsvb_execute_batch with the tile shape chosen by the caller: local_qubits per
 * shared-memory tile (7..14 for complex64, 7..13 for complex128) and register_qubits per thread
 * (4 or 5 for complex64, 3 or 4 for complex128); 0 = the engine's choice. Circuits with at most
 * local_qubits qubits run whole in one thread block; larger ones take several passes over HBM. */
int qsvb_execute_batch_ex(qsvb_ctx* ctx, const qsvb_circuit* circuits, size_t n_circuits, int dtype,
                          uint32_t local_qubits, uint32_t register_qubits, double* z0_out,
                          double* probs_out, const uint64_t* probs_offset, qsvb_plan_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* QSVB_H */
