// Internal declarations shared by the qsvb translation units (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <complex>
#include <cstdint>
#include <future>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/qsvb.h"

namespace qsvb {

using cd = std::complex<double>;

// ------------------------------------------------------------------ device bounds checks
// The context error flag (int, device memory) collects device-side failures as bits:
constexpr int kErrTimeout = 1;  // a bounded wait ran out (QSVB_E_TIMEOUT)
constexpr int kErrBounds = 2;   // a bounds check failed (checked builds only; QSVB_E_CUDA)
// A build with -DQSVB_BOUNDS_CHECK (`make -C rustatevec_b200/csrc BOUNDS=1`, which writes
// libqsvb_checked.so) range-checks the table-driven indices of the index-heavy kernels before each
// access: a failing check sets kErrBounds in the flag and the access is skipped, so a bad index
// is reported by the next synchronising call instead of touching memory it should not. In the
// ordinary build QSVB_BC(cond, err) is `true` and `cond` is not evaluated.
#if defined(__CUDACC__)
#ifdef QSVB_BOUNDS_CHECK
__device__ __forceinline__ bool bounds_ok(bool ok, int* err) {
  if (!ok) atomicOr(err, kErrBounds);
  return ok;
}
#define QSVB_BC(cond, err) ::qsvb::bounds_ok((cond), (err))
#else
#define QSVB_BC(cond, err) true
#endif
#endif

// ------------------------------------------------------------------ errors
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line);
void set_last_error(const std::string& msg);  // the message qsvb_last_error() returns on this thread
#define QSVB_CK(x)                                                        \
  do {                                                                    \
    cudaError_t _qe = (x);                                                \
    if (_qe != cudaSuccess) ::qsvb::throw_cuda(_qe, #x, __FILE__, __LINE__); \
  } while (0)
#define QSVB_REQUIRE(cond, msg)                                 \
  do {                                                          \
    if (!(cond)) throw ::qsvb::Error(QSVB_E_INVALID, (msg));    \
  } while (0)

// ------------------------------------------------------------------ sweeps (planner output)
// A sweep is one pass of one kernel over the state.
enum SweepKind : int {
  SK_1Q = 0,        // dense 2x2 on one target
  SK_CTRL = 1,      // 2x2 on one target, only where all control bits are 1 (half/quarter skip)
  SK_DIAG = 2,      // diagonal table over <= 6 qubits; "skip" qubits whose 0-half is identity
  SK_PHASE = 3,     // phase polynomial: product of many <= 2-qubit diagonal terms
  SK_DENSE = 4,     // dense 2^k x 2^k on CUDA cores
  SK_DENSE_TC = 5,  // dense 2^k x 2^k on tcgen05 tensor cores (complex64 only)
  SK_TILE = 6,      // gate program on shared-memory tiles of 2^L amplitudes (one read + one write)
  SK_NONE = 7,      // identity (dropped)
  SK_TC_CHAIN = 8,  // up to three dense 6-qubit matrices on one resident 4096-amplitude tile
                    // (tcgen05), written back with a permutation of the tile's qubits
  SK_PERMUTE = 9    // a permutation of the qubits of 4096-amplitude tiles (no arithmetic)
};
constexpr int kNumSweepKinds = 10;
constexpr int kChainMaxMats = 3;

struct Gate {  // host copy of an input gate, FP64
  uint32_t m = 0;
  uint32_t q[6] = {0, 0, 0, 0, 0, 0};
  std::vector<cd> a;  // row-major 2^m x 2^m (diag_only: the 2^m diagonal entries)
  bool diag_only = false;  // a diagonal group composed only for costing (classify_gate reads it)
};

struct PhaseTerm {
  uint32_t m;         // 1 or 2 qubits
  uint32_t q[2];
  double ang[4];      // phase angle per sub-index (bit j <-> q[j])
};

struct Sweep {
  SweepKind kind = SK_NONE;
  uint32_t m = 0;                 // qubits of the matrix (dense/diag), gate order
  uint32_t q[6] = {0, 0, 0, 0, 0, 0};
  std::vector<cd> mat;            // dense: row-major; diag: the diagonal; 1q/ctrl: 2x2
  uint32_t target = 0;            // 1q / ctrl
  uint32_t nctrl = 0;
  uint32_t ctrl[6] = {0, 0, 0, 0, 0, 0};
  std::vector<PhaseTerm> terms;   // phase polynomial
  uint64_t n_gates = 0;           // input gates covered
  // tile sweeps: the local qubit set, the gate program (1q/2q, in order) and its packed device
  // image with the launch parameters (filled by tile_prepare)
  uint64_t tile_mask = 0;
  std::vector<Gate> tile_gates;
  std::vector<uint8_t> tile_blob;
  uint32_t tile_rb = 0, tile_lbits = 0, tile_ntiles = 0;
  uint32_t tile_off_phase = 0, tile_off_prog = 0, tile_off_coef = 0;
  double tile_flops = 0;
  // chain / permutation passes: the tile's 12 state bits (ascending, bits 0..5 always among them;
  // tile position i <-> state bit chain_tbits[i]); chain_nmat matrices (64 x 64, row-major), matrix j
  // acting on tile positions chain_rows[j][0..5] (gate-index bit i <-> chain_rows[j][i]) with its
  // 64 columns ordered by chain_cols[j][0..5]; after the last matrix the amplitude at tile position
  // bit i moves to tile position bit chain_perm[i] (the pass relabels which qubit each of its
  // state bits holds)
  uint32_t chain_tbits[12] = {0};
  uint32_t chain_nmat = 0;
  uint8_t chain_rows[kChainMaxMats][6] = {};
  uint8_t chain_cols[kChainMaxMats][6] = {};
  uint8_t chain_perm[12] = {};
  std::vector<std::vector<cd>> chain_mats;
  // set by tc_chain_prepare: B operand of matrix j >= 1 K-major (1) or MN-major (0), and whether
  // the last matrix's columns 0, 1 land on output tile positions 0, 1 (16-byte epilogue stores)
  uint8_t chain_bk[kChainMaxMats] = {};
  uint8_t chain_evec = 0;
};

std::vector<Gate> gates_from_circuit(const qsvb_circuit* c);
void validate_circuit(const qsvb_circuit* c);

// Planner entry: input gates -> fused gate list (greedy/window/learned) -> classified sweeps.
std::vector<Gate> fuse_gates(const std::vector<Gate>& in, uint32_t n_qubits, const qsvb_plan_opts& o,
                             int dtype);
std::vector<Sweep> plan_sweeps(const std::vector<Gate>& in, uint32_t n_qubits,
                               const qsvb_plan_opts& o, int dtype);
Sweep classify_gate(const Gate& g);
// The product of `ops` (applied in order) on the qubit list q (index bit j <-> q[j]), in FP64.
Gate compose_gates(const std::vector<uint32_t>& q, const std::vector<const Gate*>& ops);
uint64_t gate_mask(const Gate& g);

// Host threads for planning. A thread's budget (0: the host's hardware threads, at most 16) caps
// the threads its parallel loops take; the threads a loop spawns, and the calling thread while it
// runs its share, have a budget of one, so loops nested inside them run serially. The learned
// planner gives each candidate plan's thread its share of the host.
extern thread_local uint32_t g_plan_threads;
inline size_t plan_thread_budget() {
  if (g_plan_threads) return g_plan_threads;
  return std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), 16);
}
// fn(lo, hi) over [0, n) split into contiguous ranges, on up to plan_thread_budget() threads when
// n >= min_items (else in the calling thread). Ranges are independent: results must not depend on
// the split.
template <class F> void parallel_ranges(size_t n, size_t min_items, F&& fn) {
  const size_t nth = std::min(plan_thread_budget(), n);
  if (n < min_items || nth < 2) {
    fn(size_t(0), n);
    return;
  }
  auto run = [&fn](size_t lo, size_t hi) {
    g_plan_threads = 1;
    fn(lo, hi);
  };
  std::vector<std::future<void>> fut;
  for (size_t k = 1; k < nth; ++k) fut.push_back(std::async(std::launch::async, run, n * k / nth, n * (k + 1) / nth));
  struct Restore {
    uint32_t v;
    ~Restore() { g_plan_threads = v; }
  } restore{g_plan_threads};
  g_plan_threads = 1;
  fn(size_t(0), n / nth);
  for (auto& f : fut) f.get();
}
// Tensor-core chain passes with qubit relabelling, then the permutation passes that restore every
// qubit to its own state bit (chain_planner.cpp). max_mats: matrices per pass (1..3).
std::vector<Sweep> plan_chain(const std::vector<Gate>& in, uint32_t n, uint32_t max_mats);
void sweep_costs(const std::vector<Sweep>& sw, uint32_t n, int dtype, qsvb_plan_stats* st);
qsvb_plan_opts default_opts();

// ------------------------------------------------------------------ kernel launchers
// All launchers enqueue on `s`; none synchronizes. `R` is float (complex64) or double.
struct LaunchEnv {
  cudaStream_t stream;
  int num_sms;
  int* err_flag;  // device flag a kernel sets when a bounded wait runs out
};

template <class R> void launch_init_basis(const LaunchEnv& e, R* re, R* im, uint32_t n, uint64_t basis);
template <class R> void launch_init_gaussian(const LaunchEnv& e, R* re, R* im, uint32_t n, uint64_t seed);
template <class R> void launch_scale(const LaunchEnv& e, R* re, R* im, uint32_t n, const double* d_norm);

// One sweep. `dev_mat` points to the sweep's device-side matrix block (dense kinds only) laid out
// by pack_dense_matrix(); other kinds carry their coefficients by value.
template <class R>
void launch_sweep(const LaunchEnv& e, R* re, R* im, uint32_t n, const Sweep& s, const void* dev_mat);
// Device bytes the sweep's matrix block needs (0 when the coefficients travel by value).
size_t sweep_matrix_bytes(const Sweep& s, int dtype);
void pack_sweep_matrix(const Sweep& s, int dtype, void* host_dst);

// Reductions (FP64). `partials` holds >= reduce_partials_needed() doubles; results land in
// d_out (2 doubles).
size_t reduce_partials_needed(int num_sms);
template <class R>
void launch_reduce(const LaunchEnv& e, int op, const R* re, const R* im, const R* re2, const R* im2,
                   uint32_t n, uint64_t mask, double* partials, double* d_out);
enum ReduceOp { RED_NORM = 0, RED_EXPZ = 1, RED_INNER = 2 };
template <class RA, class RB>
void launch_inner_mixed(const LaunchEnv& e, const RA* are, const RA* aim, const RB* bre, const RB* bim, uint32_t n,
                        double* partials, double* d_out);
template <class R>
void launch_probabilities(const LaunchEnv& e, const R* re, const R* im, uint64_t offset, uint64_t count,
                          void* out, int out_f64);

// Tile sweeps (batch.cu): local-qubit count for an n-qubit state (0 = state too small for tiles),
// program construction, and the launch.
uint32_t tile_local_bits(int dtype, uint32_t n);
void tile_prepare(Sweep& s, uint32_t n, int dtype);
template <class R>
void launch_tile(const LaunchEnv& e, R* re, R* im, uint32_t n, const Sweep& s, const void* dev_blob);

// Tensor-core dense sweep (complex64): implemented in tc_dense.cu.
bool tc_dense_supported(const Sweep& s, uint32_t n);
size_t tc_matrix_bytes(const Sweep& s);
void tc_pack_matrix(const Sweep& s, void* host_dst);
void launch_tc_dense(const LaunchEnv& e, float* re, float* im, uint32_t n, const Sweep& s,
                     const void* dev_mat);

// Chained tensor-core passes and tile permutations (complex64): implemented in tc_chain.cu.
// Chooses each later matrix's operand layout and row / column order (and reorders its entries) so
// that the kernel's conversions and epilogue use 16-byte shared-memory accesses; needs chain_perm.
void tc_chain_prepare(Sweep& s);
size_t tc_chain_matrix_bytes(const Sweep& s);
void tc_chain_check(const Sweep& s, uint32_t n);  // builds and validates the kernel tables (host only)
void tc_chain_pack(const Sweep& s, void* host_dst);
void launch_tc_chain(const LaunchEnv& e, float* re, float* im, uint32_t n, const Sweep& s, const void* dev_mat);
template <class R>
void launch_permute(const LaunchEnv& e, R* re, R* im, uint32_t n, const Sweep& s);

}  // namespace qsvb

// ------------------------------------------------------------------ C ABI objects
struct qsvb_state {
  uint32_t n_qubits;
  int dtype;
  int device;
  void* re;
  void* im;
};

struct qsvb_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  double* d_partials = nullptr;   // reduction partials
  double* d_result = nullptr;     // 2 doubles
  char* d_mat_ring = nullptr;     // per-apply matrix uploads
  size_t mat_ring_cap = 0;
  size_t mat_ring_pos = 0;
  char* d_exec_mats = nullptr;    // matrix block of one-shot execute calls (grow-only, reused)
  size_t exec_mats_cap = 0;
  void* d_prob = nullptr;         // probability staging chunk
  size_t prob_cap = 0;
  int* d_err = nullptr;           // device error flag (bounded waits)
  void* h_pin[2] = {nullptr, nullptr};      // pinned host ring for large device -> host copies
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
  qsvb::LaunchEnv env() const { return {stream, num_sms, d_err}; }
};

namespace qsvb {
// Large device -> host copy through the context's pinned ring: chunk k+1 crosses PCIe while the
// host copies chunk k into `dst` (pageable). `produce(k, off, len, dev_dst)` may enqueue work that
// fills a device chunk first (it returns the device pointer to copy from); pass nullptr to copy
// straight from `src`.
constexpr size_t kPinChunk = size_t(64) << 20;
void d2h_staged(qsvb_ctx* c, void* dst, const void* src, size_t bytes);
void sample_shots(qsvb_ctx* c, const qsvb_state* st, uint64_t shots, uint64_t seed, uint64_t* out);
}  // namespace qsvb

void run_batch(qsvb_ctx* c, const qsvb_circuit* circuits, size_t n_circuits, int dtype, uint32_t local_qubits,
               uint32_t register_qubits, double* z0_out, double* probs_out, const uint64_t* probs_offset,
               qsvb_plan_stats* stats);
void free_batch(qsvb_batch* b);
namespace qsvb {
uint32_t batch_max_local_bits(int dtype);
uint32_t batch_max_register_bits(int dtype);
qsvb_batch* batch_create(qsvb_ctx* c, const qsvb_circuit* circuits, size_t n, int dtype, uint32_t local_qubits,
                         uint32_t register_qubits);
void batch_run(qsvb_ctx* c, qsvb_batch* b, double* z0_out, double* probs_out, const uint64_t* probs_offset,
               qsvb_plan_stats* stats);
void batch_set_wait_budget(qsvb_ctx* c, qsvb_batch* b, uint64_t cycles);
void batch_autotune(qsvb_ctx* c, const qsvb_circuit* circuits, size_t n, int dtype, uint32_t* best_local,
                    uint32_t* best_reg, double* seconds, size_t cap, size_t* count);
}  // namespace qsvb

struct qsvb_plan {
  uint32_t n_qubits = 0;
  int dtype = 0;
  qsvb_plan_opts opts{};
  std::vector<qsvb::Sweep> sweeps;
  std::vector<size_t> mat_offset;   // byte offset of each sweep's matrix block in d_mats
  char* d_mats = nullptr;
  size_t mats_bytes = 0;
  bool owns_mats = true;            // false: d_mats is the context's execute block
  qsvb_plan_stats stats{};
  cudaGraphExec_t graph = nullptr;
  void* graph_re = nullptr;         // state the graph was captured for
  void* graph_im = nullptr;
};
