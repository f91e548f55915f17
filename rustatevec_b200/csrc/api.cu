// C ABI of the engine (include/qsvb.h): contexts, states, per-gate apply, planned execution with
// CUDA graphs, and FP64 read-outs. Every entry point catches all C++ exceptions and returns a
// status code; the message is kept per thread for qsvb_last_error().

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <future>
#include <memory>
#include <new>
#include <string>
#include <thread>

#include "cost_model.h"
#include "qsvb_internal.h"

namespace qsvb {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line) {
  const int code = e == cudaErrorMemoryAllocation ? QSVB_E_OOM : QSVB_E_CUDA;
  throw Error(code, std::string(cudaGetErrorName(e)) + " (" + cudaGetErrorString(e) + ") in " + what + " at " +
                        file + ":" + std::to_string(line));
}

namespace {

template <class F> int guarded(F&& f) {
  try {
    f();
    return QSVB_OK;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return QSVB_E_OOM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return QSVB_E_INVALID;
  } catch (...) {
    g_last_error = "unknown error";
    return QSVB_E_INVALID;
  }
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    QSVB_CK(cudaGetDevice(&prev));
    if (prev != dev) QSVB_CK(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

void check_ctx(const qsvb_ctx* c) { QSVB_REQUIRE(c != nullptr, "null context"); }

// Synchronize the context stream and surface a device-side bounded-wait timeout (the flag is
// cleared so the context stays usable).
void sync_and_check(qsvb_ctx* c) {
  QSVB_CK(cudaStreamSynchronize(c->stream));
  int flag = 0;
  QSVB_CK(cudaMemcpy(&flag, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) {
    QSVB_CK(cudaMemset(c->d_err, 0, sizeof(int)));
    if (flag & kErrBounds)
      throw Error(QSVB_E_CUDA, "a device bounds check failed (an index out of its buffer); results are invalid");
    throw Error(QSVB_E_TIMEOUT, "a device-side wait ran out of its iteration budget; results are invalid");
  }
}
void check_state(const qsvb_ctx* c, const qsvb_state* s) {
  check_ctx(c);
  QSVB_REQUIRE(s != nullptr, "null state");
  QSVB_REQUIRE(s->device == c->device, "state belongs to another device");
}

size_t state_bytes(const qsvb_state* s) { return (s->dtype == QSVB_C128 ? 8u : 4u) * (size_t(1) << s->n_qubits); }

template <class F> void by_dtype(int dtype, F&& f) {
  if (dtype == QSVB_C128) f(double{});
  else f(float{});
}

// Upload a block to the context's matrix ring (stream-ordered; the source is pageable host memory,
// which the runtime stages before cudaMemcpyAsync returns, so the caller's buffer can be reused).
void* ring_upload(qsvb_ctx* c, const void* src, size_t bytes) {
  const size_t need = (bytes + 255) & ~size_t(255);
  if (need > c->mat_ring_cap) {
    QSVB_CK(cudaStreamSynchronize(c->stream));
    if (c->d_mat_ring) QSVB_CK(cudaFree(c->d_mat_ring));
    c->mat_ring_cap = std::max(need, size_t(1) << 20);
    QSVB_CK(cudaMalloc(&c->d_mat_ring, c->mat_ring_cap));
    c->mat_ring_pos = 0;
  }
  if (c->mat_ring_pos + need > c->mat_ring_cap) c->mat_ring_pos = 0;
  char* dst = c->d_mat_ring + c->mat_ring_pos;
  c->mat_ring_pos += need;
  QSVB_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
  return dst;
}

void run_sweep(qsvb_ctx* c, qsvb_state* st, const Sweep& s, const void* dev_mat) {
  by_dtype(st->dtype, [&](auto r) {
    using R = decltype(r);
    launch_sweep<R>(c->env(), static_cast<R*>(st->re), static_cast<R*>(st->im), st->n_qubits, s, dev_mat);
  });
}

// exec_block: the plan is run once and freed by the caller before the context's next call (one-shot
// execute); its matrices then go into the context's reusable block instead of an allocation of
// their own, so a one-shot call allocates and frees nothing on the device once the block is large
// enough (a cudaFree can stall the host for tens to hundreds of milliseconds).
qsvb_plan* build_plan(qsvb_ctx* c, const qsvb_circuit* circ, int dtype, const qsvb_plan_opts* opts,
                      bool exec_block) {
  validate_circuit(circ);
  QSVB_REQUIRE(dtype == QSVB_C64 || dtype == QSVB_C128, "dtype must be QSVB_C64 or QSVB_C128");
  std::unique_ptr<qsvb_plan> p(new qsvb_plan);
  p->n_qubits = circ->n_qubits;
  p->dtype = dtype;
  p->opts = opts ? *opts : default_opts();
  p->sweeps = plan_sweeps(gates_from_circuit(circ), circ->n_qubits, p->opts, dtype);
  p->stats.n_gates_in = circ->n_gates;
  sweep_costs(p->sweeps, circ->n_qubits, dtype, &p->stats);
  // one device block holding every sweep's matrix, uploaded once
  size_t total = 0;
  for (const Sweep& s : p->sweeps) {
    p->mat_offset.push_back(total);
    total += (sweep_matrix_bytes(s, dtype) + 255) & ~size_t(255);
  }
  p->mats_bytes = total;
  if (total) {
    std::vector<char> host(total, 0);
    // each sweep packs into its own range (the tensor-core bf16 hi/lo images take about 50 us a
    // matrix): large plans pack on several host threads
    auto pack_range = [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; ++i)
        if (sweep_matrix_bytes(p->sweeps[i], dtype)) pack_sweep_matrix(p->sweeps[i], dtype, host.data() + p->mat_offset[i]);
    };
    const size_t ns = p->sweeps.size();
    const size_t nth = std::min<size_t>({size_t(std::max(1u, std::thread::hardware_concurrency())), size_t(8), ns});
    if (total < (size_t(1) << 20) || nth < 2) {
      pack_range(0, ns);
    } else {
      std::vector<std::future<void>> fut;
      for (size_t t = 1; t < nth; ++t) fut.push_back(std::async(std::launch::async, pack_range, ns * t / nth, ns * (t + 1) / nth));
      pack_range(0, ns / nth);
      for (auto& f : fut) f.get();
    }
    if (exec_block) {
      if (c->exec_mats_cap < total) {
        QSVB_CK(cudaStreamSynchronize(c->stream));  // the previous call's kernels may still read it
        if (c->d_exec_mats) QSVB_CK(cudaFree(c->d_exec_mats));
        c->d_exec_mats = nullptr;
        c->exec_mats_cap = 0;
        QSVB_CK(cudaMalloc(&c->d_exec_mats, total));
        c->exec_mats_cap = total;
      }
      p->d_mats = c->d_exec_mats;
      p->owns_mats = false;
      // stream-ordered after every earlier use of the block on this context's stream
      QSVB_CK(cudaMemcpyAsync(p->d_mats, host.data(), total, cudaMemcpyHostToDevice, c->stream));
      QSVB_CK(cudaStreamSynchronize(c->stream));  // `host` is pageable and about to go away
    } else {
      QSVB_CK(cudaMalloc(&p->d_mats, total));
      QSVB_CK(cudaMemcpy(p->d_mats, host.data(), total, cudaMemcpyHostToDevice));
    }
  }
  return p.release();
}

void launch_plan(qsvb_ctx* c, qsvb_plan* p, qsvb_state* st) {
  for (size_t i = 0; i < p->sweeps.size(); ++i) {
    const void* m = sweep_matrix_bytes(p->sweeps[i], p->dtype) ? p->d_mats + p->mat_offset[i] : nullptr;
    run_sweep(c, st, p->sweeps[i], m);
  }
}

void run_plan(qsvb_ctx* c, qsvb_plan* p, qsvb_state* st) {
  QSVB_REQUIRE(st->n_qubits == p->n_qubits, "plan and state qubit counts differ");
  QSVB_REQUIRE(st->dtype == p->dtype, "plan and state precisions differ");
  if (!p->opts.use_graph || p->sweeps.empty()) {
    launch_plan(c, p, st);
    return;
  }
  if (p->graph && (p->graph_re != st->re || p->graph_im != st->im)) {
    QSVB_CK(cudaGraphExecDestroy(p->graph));
    p->graph = nullptr;
  }
  if (!p->graph) {
    cudaGraph_t g = nullptr;
    QSVB_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    try {
      launch_plan(c, p, st);
    } catch (...) {
      cudaStreamEndCapture(c->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    QSVB_CK(cudaStreamEndCapture(c->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&p->graph, g, 0);
    cudaGraphDestroy(g);
    QSVB_CK(e);
    p->graph_re = st->re;
    p->graph_im = st->im;
  }
  QSVB_CK(cudaGraphLaunch(p->graph, c->stream));
}

void free_plan(qsvb_plan* p) {
  if (!p) return;
  if (p->graph) cudaGraphExecDestroy(p->graph);
  if (p->d_mats && p->owns_mats) cudaFree(p->d_mats);
  delete p;
}

double reduce(qsvb_ctx* c, int op, const qsvb_state* a, const qsvb_state* b, uint64_t mask, double* second) {
  by_dtype(a->dtype, [&](auto r) {
    using R = decltype(r);
    launch_reduce<R>(c->env(), op, static_cast<const R*>(a->re), static_cast<const R*>(a->im),
                     b ? static_cast<const R*>(b->re) : nullptr, b ? static_cast<const R*>(b->im) : nullptr,
                     a->n_qubits, mask, c->d_partials, c->d_result);
  });
  double h[2];
  QSVB_CK(cudaMemcpyAsync(h, c->d_result, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  sync_and_check(c);
  if (second) *second = h[1];
  return h[0];
}

}  // namespace
}  // namespace qsvb

using namespace qsvb;

extern "C" {

const char* qsvb_last_error(void) { return g_last_error.c_str(); }

const char* qsvb_version(void) { return "qsvb 0.1 sm_100a"; }

int qsvb_create(int device_ordinal, qsvb_ctx** out) {
  return guarded([&] {
    QSVB_REQUIRE(out != nullptr, "null output pointer");
    int ndev = 0;
    QSVB_CK(cudaGetDeviceCount(&ndev));
    QSVB_REQUIRE(device_ordinal >= 0 && device_ordinal < ndev, "no such CUDA device");
    DeviceGuard dg(device_ordinal);
    cudaDeviceProp prop{};
    QSVB_CK(cudaGetDeviceProperties(&prop, device_ordinal));
    if (prop.major != 10)
      throw Error(QSVB_E_UNSUPPORTED, std::string("this build targets sm_100a (B200); device is ") + prop.name);
    std::unique_ptr<qsvb_ctx> c(new qsvb_ctx);
    c->device = device_ordinal;
    c->num_sms = prop.multiProcessorCount;
    QSVB_CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    QSVB_CK(cudaMalloc(&c->d_partials, reduce_partials_needed(c->num_sms) * sizeof(double)));
    QSVB_CK(cudaMalloc(&c->d_result, 2 * sizeof(double)));
    QSVB_CK(cudaMalloc(&c->d_err, sizeof(int)));
    QSVB_CK(cudaMemset(c->d_err, 0, sizeof(int)));
    *out = c.release();
  });
}

int qsvb_destroy(qsvb_ctx* c) {
  return guarded([&] {
    if (!c) return;
    DeviceGuard dg(c->device);
    cudaStreamSynchronize(c->stream);
    if (c->d_partials) cudaFree(c->d_partials);
    if (c->d_result) cudaFree(c->d_result);
    if (c->d_mat_ring) cudaFree(c->d_mat_ring);
    if (c->d_exec_mats) cudaFree(c->d_exec_mats);
    if (c->d_prob) cudaFree(c->d_prob);
    if (c->d_err) cudaFree(c->d_err);
    for (int i = 0; i < 2; ++i) {
      if (c->h_pin[i]) cudaFreeHost(c->h_pin[i]);
      if (c->pin_ev[i]) cudaEventDestroy(c->pin_ev[i]);
    }
    cudaStreamDestroy(c->stream);
    delete c;
  });
}

int qsvb_stream(qsvb_ctx* c, void** out) {
  return guarded([&] {
    check_ctx(c);
    QSVB_REQUIRE(out != nullptr, "null output pointer");
    *out = reinterpret_cast<void*>(c->stream);
  });
}

int qsvb_synchronize(qsvb_ctx* c) {
  return guarded([&] {
    check_ctx(c);
    DeviceGuard dg(c->device);
    sync_and_check(c);
  });
}

int qsvb_state_alloc(qsvb_ctx* c, uint32_t n, int dtype, qsvb_state** out) {
  return guarded([&] {
    check_ctx(c);
    QSVB_REQUIRE(out != nullptr, "null output pointer");
    QSVB_REQUIRE(n >= 1 && n <= QSVB_MAX_QUBITS, "qubit count must be 1..34");
    QSVB_REQUIRE(dtype == QSVB_C64 || dtype == QSVB_C128, "dtype must be QSVB_C64 or QSVB_C128");
    DeviceGuard dg(c->device);
    std::unique_ptr<qsvb_state> s(new qsvb_state{n, dtype, c->device, nullptr, nullptr});
    const size_t bytes = state_bytes(s.get());
    size_t free_b = 0, total_b = 0;
    QSVB_CK(cudaMemGetInfo(&free_b, &total_b));
    if (2 * bytes > free_b)
      throw Error(QSVB_E_OOM, "state of " + std::to_string(n) + " qubits needs " + std::to_string(2 * bytes) +
                                  " bytes; " + std::to_string(free_b) + " free");
    cudaError_t e = cudaMalloc(&s->re, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&s->im, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      if (s->re) cudaFree(s->re);
      throw Error(QSVB_E_OOM, std::string("state allocation failed: ") + cudaGetErrorString(e));
    }
    *out = s.release();
  });
}

int qsvb_state_free(qsvb_ctx* c, qsvb_state* s) {
  return guarded([&] {
    if (!s) return;
    check_state(c, s);
    DeviceGuard dg(c->device);
    QSVB_CK(cudaStreamSynchronize(c->stream));
    cudaFree(s->re);
    cudaFree(s->im);
    delete s;
  });
}

int qsvb_state_info(const qsvb_state* s, uint32_t* n, int* dtype, void** re, void** im) {
  return guarded([&] {
    QSVB_REQUIRE(s != nullptr, "null state");
    if (n) *n = s->n_qubits;
    if (dtype) *dtype = s->dtype;
    if (re) *re = s->re;
    if (im) *im = s->im;
  });
}

int qsvb_init_basis(qsvb_ctx* c, qsvb_state* s, uint64_t basis) {
  return guarded([&] {
    check_state(c, s);
    QSVB_REQUIRE(basis < (uint64_t(1) << s->n_qubits), "basis index out of range");
    DeviceGuard dg(c->device);
    by_dtype(s->dtype, [&](auto r) {
      using R = decltype(r);
      launch_init_basis<R>(c->env(), static_cast<R*>(s->re), static_cast<R*>(s->im), s->n_qubits, basis);
    });
  });
}

int qsvb_upload(qsvb_ctx* c, qsvb_state* s, const void* re, const void* im) {
  return guarded([&] {
    check_state(c, s);
    QSVB_REQUIRE(re && im, "null host buffer");
    DeviceGuard dg(c->device);
    const size_t b = state_bytes(s);
    QSVB_CK(cudaMemcpyAsync(s->re, re, b, cudaMemcpyHostToDevice, c->stream));
    QSVB_CK(cudaMemcpyAsync(s->im, im, b, cudaMemcpyHostToDevice, c->stream));
    QSVB_CK(cudaStreamSynchronize(c->stream));
  });
}

int qsvb_init_gaussian(qsvb_ctx* c, qsvb_state* s, uint64_t seed) {
  return guarded([&] {
    check_state(c, s);
    DeviceGuard dg(c->device);
    by_dtype(s->dtype, [&](auto r) {
      using R = decltype(r);
      R* re = static_cast<R*>(s->re);
      R* im = static_cast<R*>(s->im);
      launch_init_gaussian<R>(c->env(), re, im, s->n_qubits, seed);
      launch_reduce<R>(c->env(), RED_NORM, re, im, nullptr, nullptr, s->n_qubits, 0, c->d_partials, c->d_result);
      launch_scale<R>(c->env(), re, im, s->n_qubits, c->d_result);
    });
  });
}

int qsvb_apply(qsvb_ctx* c, qsvb_state* s, const double* matrix, const uint32_t* qubits, uint32_t m) {
  return guarded([&] {
    check_state(c, s);
    QSVB_REQUIRE(matrix && qubits, "null matrix or qubit list");
    qsvb_gate g{};
    g.n_qubits = m;
    QSVB_REQUIRE(m >= 1 && m <= QSVB_MAX_GATE_QUBITS, "gate arity must be 1..6");
    for (uint32_t j = 0; j < m; ++j) g.qubits[j] = qubits[j];
    g.matrix = matrix;
    qsvb_circuit circ{s->n_qubits, 1, &g};
    validate_circuit(&circ);
    DeviceGuard dg(c->device);
    Sweep sw = classify_gate(gates_from_circuit(&circ)[0]);
    if (sw.kind == SK_NONE) return;
    const size_t mb = sweep_matrix_bytes(sw, s->dtype);
    const void* dm = nullptr;
    if (mb) {
      std::vector<char> host(mb);
      pack_sweep_matrix(sw, s->dtype, host.data());
      dm = ring_upload(c, host.data(), mb);
    }
    run_sweep(c, s, sw, dm);
  });
}

int qsvb_plan_create(qsvb_ctx* c, const qsvb_circuit* circ, int dtype, const qsvb_plan_opts* opts, qsvb_plan** out) {
  return guarded([&] {
    check_ctx(c);
    QSVB_REQUIRE(out != nullptr, "null output pointer");
    DeviceGuard dg(c->device);
    *out = build_plan(c, circ, dtype, opts, false);
  });
}

int qsvb_plan_run(qsvb_ctx* c, qsvb_plan* p, qsvb_state* s) {
  return guarded([&] {
    check_state(c, s);
    QSVB_REQUIRE(p != nullptr, "null plan");
    DeviceGuard dg(c->device);
    run_plan(c, p, s);
  });
}

int qsvb_plan_stats_get(const qsvb_plan* p, qsvb_plan_stats* out) {
  return guarded([&] {
    QSVB_REQUIRE(p && out, "null plan or output");
    *out = p->stats;
  });
}

int qsvb_plan_sweep_info(const qsvb_plan* p, size_t i, qsvb_sweep_info* out) {
  return guarded([&] {
    QSVB_REQUIRE(p && out, "null plan or output");
    QSVB_REQUIRE(i < p->sweeps.size(), "sweep index out of range");
    const Sweep& s = p->sweeps[i];
    *out = qsvb_sweep_info{};
    out->kind = uint32_t(s.kind);
    out->n_qubits = s.m;
    for (uint32_t j = 0; j < QSVB_MAX_GATE_QUBITS; ++j) {
      out->qubits[j] = s.q[j];
      out->ctrl[j] = s.ctrl[j];
    }
    out->target = s.target;
    out->n_ctrl = s.nctrl;
    out->n_terms = uint32_t(s.terms.size());
    out->n_gates = s.n_gates;
    if (s.kind == SK_TC_CHAIN || s.kind == SK_PERMUTE) {
      out->n_qubits = s.chain_nmat;
      for (uint32_t j = 0; j < 6; ++j) out->qubits[j] = s.chain_tbits[6 + j];
    }
    qsvb_plan_stats one{};
    sweep_costs(std::vector<Sweep>{s}, p->n_qubits, p->dtype, &one);
    out->algorithmic_bytes = one.algorithmic_bytes;
    out->flops = one.flops;
    sweep_features(s, p->n_qubits, p->dtype, out->features);
  });
}

int qsvb_plan_profile(qsvb_ctx* c, qsvb_plan* p, qsvb_state* s, int reps, double* out) {
  return guarded([&] {
    check_state(c, s);
    QSVB_REQUIRE(p && out, "null plan or output");
    QSVB_REQUIRE(reps >= 1 && reps <= 1000, "reps must be 1..1000");
    QSVB_REQUIRE(s->n_qubits == p->n_qubits && s->dtype == p->dtype, "plan and state differ");
    DeviceGuard dg(c->device);
    cudaEvent_t e0, e1;
    QSVB_CK(cudaEventCreate(&e0));
    QSVB_CK(cudaEventCreate(&e1));
    try {
      for (size_t i = 0; i < p->sweeps.size(); ++i) {
        const void* m = sweep_matrix_bytes(p->sweeps[i], p->dtype) ? p->d_mats + p->mat_offset[i] : nullptr;
        run_sweep(c, s, p->sweeps[i], m);  // warm-up launch
        QSVB_CK(cudaEventRecord(e0, c->stream));
        for (int r = 0; r < reps; ++r) run_sweep(c, s, p->sweeps[i], m);
        QSVB_CK(cudaEventRecord(e1, c->stream));
        QSVB_CK(cudaEventSynchronize(e1));
        float ms = 0;
        QSVB_CK(cudaEventElapsedTime(&ms, e0, e1));
        out[i] = double(ms) * 1e-3 / reps;
      }
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  });
}

int qsvb_plan_free(qsvb_ctx* c, qsvb_plan* p) {
  return guarded([&] {
    if (!p) return;
    check_ctx(c);
    DeviceGuard dg(c->device);
    QSVB_CK(cudaStreamSynchronize(c->stream));
    free_plan(p);
  });
}

int qsvb_execute(qsvb_ctx* c, qsvb_state* s, const qsvb_circuit* circ, const qsvb_plan_opts* opts,
                 qsvb_plan_stats* stats) {
  return guarded([&] {
    check_state(c, s);
    QSVB_REQUIRE(circ != nullptr, "null circuit");
    QSVB_REQUIRE(circ->n_qubits == s->n_qubits, "circuit and state qubit counts differ");
    DeviceGuard dg(c->device);
    std::unique_ptr<qsvb_plan, void (*)(qsvb_plan*)> p(build_plan(c, circ, s->dtype, opts, true), free_plan);
    // one run: launched directly, so the first sweep starts while later ones are still queued
    p->opts.use_graph = 0;
    run_plan(c, p.get(), s);
    if (stats) *stats = p->stats;
    // the plan's device matrices and graph must outlive the queued work
    sync_and_check(c);
  });
}

int qsvb_plan_dry_run(const qsvb_circuit* circ, int dtype, const qsvb_plan_opts* opts, qsvb_plan_stats* stats) {
  return guarded([&] {
    validate_circuit(circ);
    QSVB_REQUIRE(dtype == QSVB_C64 || dtype == QSVB_C128, "dtype must be QSVB_C64 or QSVB_C128");
    QSVB_REQUIRE(stats != nullptr, "null output");
    const qsvb_plan_opts o = opts ? *opts : default_opts();
    const std::vector<Sweep> sw = plan_sweeps(gates_from_circuit(circ), circ->n_qubits, o, dtype);
    *stats = qsvb_plan_stats{};
    stats->n_gates_in = circ->n_gates;
    sweep_costs(sw, circ->n_qubits, dtype, stats);
  });
}

int qsvb_fuse(const qsvb_circuit* circ, const qsvb_plan_opts* opts, qsvb_gate* out_gates, size_t* n_out,
              double* out_mats, size_t cap) {
  return guarded([&] {
    validate_circuit(circ);
    QSVB_REQUIRE(n_out != nullptr, "null count pointer");
    const qsvb_plan_opts o = opts ? *opts : default_opts();
    std::vector<Gate> fused;
    if (o.planner == QSVB_PLAN_LEARNED)
      fused = learned_fuse(gates_from_circuit(circ), circ->n_qubits, o, QSVB_C64);
    else
      fused = fuse_gates(gates_from_circuit(circ), circ->n_qubits, o, QSVB_C64);
    if (!out_gates) {
      *n_out = fused.size();
      return;
    }
    QSVB_REQUIRE(*n_out >= fused.size(), "output gate array too small");
    size_t need = 0;
    for (const Gate& g : fused) need += 2 * g.a.size();
    QSVB_REQUIRE(cap >= need, "output matrix buffer too small");
    size_t mo = 0;
    for (size_t i = 0; i < fused.size(); ++i) {
      qsvb_gate& og = out_gates[i];
      og.n_qubits = fused[i].m;
      for (uint32_t j = 0; j < QSVB_MAX_GATE_QUBITS; ++j) og.qubits[j] = j < fused[i].m ? fused[i].q[j] : 0;
      og.matrix = out_mats + mo;
      for (const cd& v : fused[i].a) {
        out_mats[mo++] = v.real();
        out_mats[mo++] = v.imag();
      }
    }
    *n_out = fused.size();
  });
}

int qsvb_download(qsvb_ctx* c, const qsvb_state* s, void* re, void* im) {
  return guarded([&] {
    check_state(c, s);
    QSVB_REQUIRE(re && im, "null host buffer");
    DeviceGuard dg(c->device);
    const size_t b = state_bytes(s);
    QSVB_CK(cudaMemcpyAsync(re, s->re, b, cudaMemcpyDeviceToHost, c->stream));
    QSVB_CK(cudaMemcpyAsync(im, s->im, b, cudaMemcpyDeviceToHost, c->stream));
    sync_and_check(c);  // also reports a failure flagged by earlier device work
  });
}

int qsvb_amplitude(qsvb_ctx* c, const qsvb_state* s, uint64_t index, double out[2]) {
  return guarded([&] {
    check_state(c, s);
    QSVB_REQUIRE(out != nullptr, "null output");
    QSVB_REQUIRE(index < (uint64_t(1) << s->n_qubits), "amplitude index out of range");
    DeviceGuard dg(c->device);
    if (s->dtype == QSVB_C128) {
      QSVB_CK(cudaMemcpyAsync(&out[0], static_cast<double*>(s->re) + index, 8, cudaMemcpyDeviceToHost, c->stream));
      QSVB_CK(cudaMemcpyAsync(&out[1], static_cast<double*>(s->im) + index, 8, cudaMemcpyDeviceToHost, c->stream));
      sync_and_check(c);  // also reports a failure flagged by earlier device work
    } else {
      float v[2];
      QSVB_CK(cudaMemcpyAsync(&v[0], static_cast<float*>(s->re) + index, 4, cudaMemcpyDeviceToHost, c->stream));
      QSVB_CK(cudaMemcpyAsync(&v[1], static_cast<float*>(s->im) + index, 4, cudaMemcpyDeviceToHost, c->stream));
      sync_and_check(c);  // also reports a failure flagged by earlier device work
      out[0] = v[0];
      out[1] = v[1];
    }
  });
}

}  // extern "C"

namespace qsvb {
namespace {
void ensure_pinned(qsvb_ctx* c) {
  for (int i = 0; i < 2; ++i) {
    if (!c->h_pin[i]) QSVB_CK(cudaHostAlloc(&c->h_pin[i], kPinChunk, cudaHostAllocDefault));
    if (!c->pin_ev[i]) QSVB_CK(cudaEventCreateWithFlags(&c->pin_ev[i], cudaEventDisableTiming));
  }
}

// host copy of one staged chunk, split over a few threads (one thread moves ~10 GB/s, less while
// it first touches fresh pages of the destination)
void host_copy(void* dst, const void* src, size_t bytes) {
  constexpr int kThreads = 8;
  if (bytes < (size_t(4) << 20)) {
    std::memcpy(dst, src, bytes);
    return;
  }
  std::thread th[kThreads - 1];
  const size_t part = (bytes / kThreads + 63) & ~size_t(63);
  for (int t = 1; t < kThreads; ++t) {
    const size_t off = std::min(bytes, part * t), len = std::min(bytes - off, part);
    th[t - 1] = std::thread([=] { std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, len); });
  }
  std::memcpy(dst, src, std::min(bytes, part));
  for (auto& t : th) t.join();
}
}  // namespace

void d2h_staged(qsvb_ctx* c, void* dst, const void* src, size_t bytes) {
  if (bytes <= (size_t(4) << 20)) {
    QSVB_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    QSVB_CK(cudaStreamSynchronize(c->stream));
    return;
  }
  ensure_pinned(c);
  const size_t n = (bytes + kPinChunk - 1) / kPinChunk;
  auto issue = [&](size_t k) {
    const size_t off = k * kPinChunk, len = std::min(kPinChunk, bytes - off);
    QSVB_CK(cudaMemcpyAsync(c->h_pin[k & 1], static_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost,
                            c->stream));
    QSVB_CK(cudaEventRecord(c->pin_ev[k & 1], c->stream));
  };
  issue(0);
  for (size_t k = 0; k < n; ++k) {
    if (k + 1 < n) issue(k + 1);  // its buffer held chunk k-1, copied out in the previous step
    QSVB_CK(cudaEventSynchronize(c->pin_ev[k & 1]));
    const size_t off = k * kPinChunk;
    host_copy(static_cast<char*>(dst) + off, c->h_pin[k & 1], std::min(kPinChunk, bytes - off));
  }
}
}  // namespace qsvb

extern "C" {
int qsvb_probabilities(qsvb_ctx* c, const qsvb_state* s, void* out, int out_dtype) {
  return guarded([&] {
    check_state(c, s);
    QSVB_REQUIRE(out != nullptr, "null output");
    QSVB_REQUIRE(out_dtype == QSVB_C64 || out_dtype == QSVB_C128, "out_dtype must be QSVB_C64 or QSVB_C128");
    DeviceGuard dg(c->device);
    const uint64_t dim = uint64_t(1) << s->n_qubits;
    const size_t esz = out_dtype == QSVB_C128 ? 8 : 4;
    // chunks of one pinned buffer: chunk k is computed and crosses PCIe while the host copies
    // chunk k-1 into `out`
    const uint64_t chunk = std::min<uint64_t>(dim, kPinChunk / esz);
    if (c->prob_cap < chunk * esz) {
      QSVB_CK(cudaStreamSynchronize(c->stream));
      if (c->d_prob) QSVB_CK(cudaFree(c->d_prob));
      c->d_prob = nullptr;
      QSVB_CK(cudaMalloc(&c->d_prob, chunk * esz));
      c->prob_cap = chunk * esz;
    }
    ensure_pinned(c);
    const uint64_t nchunk = (dim + chunk - 1) / chunk;
    for (uint64_t k = 0; k <= nchunk; ++k) {
      if (k < nchunk) {
        const uint64_t off = k * chunk, cnt = std::min(chunk, dim - off);
        by_dtype(s->dtype, [&](auto r) {
          using R = decltype(r);
          launch_probabilities<R>(c->env(), static_cast<const R*>(s->re), static_cast<const R*>(s->im), off, cnt,
                                  c->d_prob, out_dtype == QSVB_C128);
        });
        QSVB_CK(cudaMemcpyAsync(c->h_pin[k & 1], c->d_prob, cnt * esz, cudaMemcpyDeviceToHost, c->stream));
        QSVB_CK(cudaEventRecord(c->pin_ev[k & 1], c->stream));
      }
      if (k >= 1) {
        const uint64_t j = k - 1, off = j * chunk, cnt = std::min(chunk, dim - off);
        QSVB_CK(cudaEventSynchronize(c->pin_ev[j & 1]));
        host_copy(static_cast<char*>(out) + off * esz, c->h_pin[j & 1], cnt * esz);
      }
    }
    sync_and_check(c);
  });
}

int qsvb_sample(qsvb_ctx* c, const qsvb_state* s, uint64_t shots, uint64_t seed, uint64_t* out) {
  return guarded([&] {
    check_state(c, s);
    DeviceGuard dg(c->device);
    sample_shots(c, s, shots, seed, out);
  });
}

int qsvb_expectation_z(qsvb_ctx* c, const qsvb_state* s, uint64_t mask, double* out) {
  return guarded([&] {
    check_state(c, s);
    QSVB_REQUIRE(out != nullptr, "null output");
    DeviceGuard dg(c->device);
    *out = reduce(c, RED_EXPZ, s, nullptr, mask, nullptr);
  });
}

int qsvb_norm_sqr(qsvb_ctx* c, const qsvb_state* s, double* out) {
  return guarded([&] {
    check_state(c, s);
    QSVB_REQUIRE(out != nullptr, "null output");
    DeviceGuard dg(c->device);
    *out = reduce(c, RED_NORM, s, nullptr, 0, nullptr);
  });
}

int qsvb_inner_product(qsvb_ctx* c, const qsvb_state* a, const qsvb_state* b, double out[2]) {
  return guarded([&] {
    check_state(c, a);
    check_state(c, b);
    QSVB_REQUIRE(out != nullptr, "null output");
    QSVB_REQUIRE(a->n_qubits == b->n_qubits, "states differ in qubit count");
    DeviceGuard dg(c->device);
    if (a->dtype == b->dtype) {
      out[0] = reduce(c, RED_INNER, a, b, 0, &out[1]);
      return;
    }
    // mixed precision: complex64 against complex128, accumulated in FP64
    if (a->dtype == QSVB_C64)
      launch_inner_mixed<float, double>(c->env(), static_cast<const float*>(a->re), static_cast<const float*>(a->im),
                                        static_cast<const double*>(b->re), static_cast<const double*>(b->im),
                                        a->n_qubits, c->d_partials, c->d_result);
    else
      launch_inner_mixed<double, float>(c->env(), static_cast<const double*>(a->re), static_cast<const double*>(a->im),
                                        static_cast<const float*>(b->re), static_cast<const float*>(b->im),
                                        a->n_qubits, c->d_partials, c->d_result);
    QSVB_CK(cudaMemcpyAsync(out, c->d_result, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    sync_and_check(c);  // also reports a failure flagged by earlier device work
  });
}

int qsvb_fidelity(qsvb_ctx* c, const qsvb_state* a, const qsvb_state* b, double* out) {
  return guarded([&] {
    QSVB_REQUIRE(out != nullptr, "null output");
    double ip[2];
    const int rc = qsvb_inner_product(c, a, b, ip);
    if (rc) throw Error(rc, g_last_error);
    *out = ip[0] * ip[0] + ip[1] * ip[1];
  });
}

int qsvb_execute_batch(qsvb_ctx* c, const qsvb_circuit* circuits, size_t n_circuits, int dtype, double* z0_out,
                       double* probs_out, const uint64_t* probs_offset, qsvb_plan_stats* stats) {
  return guarded([&] {
    check_ctx(c);
    DeviceGuard dg(c->device);
    run_batch(c, circuits, n_circuits, dtype, 0, 0, z0_out, probs_out, probs_offset, stats);
  });
}

int qsvb_batch_create(qsvb_ctx* c, const qsvb_circuit* circuits, size_t n_circuits, int dtype, uint32_t local_qubits,
                      uint32_t register_qubits, qsvb_batch** out) {
  return guarded([&] {
    check_ctx(c);
    QSVB_REQUIRE(out != nullptr, "null output");
    *out = nullptr;
    DeviceGuard dg(c->device);
    *out = qsvb::batch_create(c, circuits, n_circuits, dtype, local_qubits, register_qubits);
  });
}

int qsvb_batch_run(qsvb_ctx* c, qsvb_batch* b, double* z0_out, double* probs_out, const uint64_t* probs_offset,
                   qsvb_plan_stats* stats) {
  return guarded([&] {
    check_ctx(c);
    DeviceGuard dg(c->device);
    qsvb::batch_run(c, b, z0_out, probs_out, probs_offset, stats);
  });
}

int qsvb_batch_set_wait_budget(qsvb_ctx* c, qsvb_batch* b, uint64_t cycles) {
  return guarded([&] {
    check_ctx(c);
    DeviceGuard dg(c->device);
    qsvb::batch_set_wait_budget(c, b, cycles);
  });
}

int qsvb_batch_free(qsvb_ctx* c, qsvb_batch* b) {
  return guarded([&] {
    check_ctx(c);
    DeviceGuard dg(c->device);
    free_batch(b);
  });
}

int qsvb_batch_autotune(qsvb_ctx* c, const qsvb_circuit* circuits, size_t n_circuits, int dtype,
                        uint32_t* best_local, uint32_t* best_register, double* seconds, size_t cap, size_t* count) {
  return guarded([&] {
    check_ctx(c);
    QSVB_REQUIRE(best_local != nullptr && best_register != nullptr, "null output");
    DeviceGuard dg(c->device);
    qsvb::batch_autotune(c, circuits, n_circuits, dtype, best_local, best_register, seconds, cap, count);
  });
}

int qsvb_execute_batch_ex(qsvb_ctx* c, const qsvb_circuit* circuits, size_t n_circuits, int dtype,
                          uint32_t local_qubits, uint32_t register_qubits, double* z0_out, double* probs_out,
                          const uint64_t* probs_offset, qsvb_plan_stats* stats) {
  return guarded([&] {
    check_ctx(c);
    DeviceGuard dg(c->device);
    run_batch(c, circuits, n_circuits, dtype, local_qubits, register_qubits, z0_out, probs_out, probs_offset, stats);
  });
}

}  // extern "C"
