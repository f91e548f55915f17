// Autotuner: times candidate sweeps on the device and returns (features, seconds) records, the
// training data of the MLP cost model (mlp.cu) and the evidence the planner's engine choice rests
// on. Candidates cover every sweep kind, k = 1..6, CUDA-core and tensor-core dense engines, and the
// qubit placements that change a kernel's memory pattern (low / high / mid / two runs / scattered /
// one low bit).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "cost_model.h"
#include "qsvb_internal.h"

namespace qsvb {
namespace {

std::vector<cd> haar(uint32_t k, std::mt19937_64& rng) {
  const size_t d = size_t(1) << k;
  std::normal_distribution<double> nd;
  std::vector<cd> a(d * d);
  for (auto& x : a) x = cd(nd(rng), nd(rng));
  // Gram-Schmidt on columns
  for (size_t c = 0; c < d; ++c) {
    for (size_t p = 0; p < c; ++p) {
      cd dot = 0;
      for (size_t r = 0; r < d; ++r) dot += std::conj(a[r * d + p]) * a[r * d + c];
      for (size_t r = 0; r < d; ++r) a[r * d + c] -= dot * a[r * d + p];
    }
    double nrm = 0;
    for (size_t r = 0; r < d; ++r) nrm += std::norm(a[r * d + c]);
    nrm = std::sqrt(nrm);
    for (size_t r = 0; r < d; ++r) a[r * d + c] /= nrm;
  }
  return a;
}

std::vector<std::vector<uint32_t>> placements(uint32_t k, uint32_t n) {
  std::vector<std::vector<uint32_t>> out;
  auto range = [](uint32_t a, uint32_t k) {
    std::vector<uint32_t> v;
    for (uint32_t i = 0; i < k; ++i) v.push_back(a + i);
    return v;
  };
  out.push_back(range(0, k));
  out.push_back(range(n - k, k));
  if (n >= k + 8) out.push_back(range(3, k));
  if (n >= 2 * k + 4 && k >= 2) {  // two runs (brickwork-window shape)
    std::vector<uint32_t> v = range(5, k / 2);
    for (uint32_t i = 0; i < k - k / 2; ++i) v.push_back(11 + i);
    out.push_back(v);
  }
  if (n >= 2 * k + 8) {  // scattered
    std::vector<uint32_t> v;
    for (uint32_t i = 0; i < k; ++i) v.push_back(7 + 2 * i);
    out.push_back(v);
  }
  if (k >= 2 && n >= k + 10) {  // bit 0 in the gate, bit 1 not
    std::vector<uint32_t> v = {0};
    for (uint32_t i = 1; i < k; ++i) v.push_back(8 + i);
    out.push_back(v);
  }
  return out;
}

}  // namespace

std::vector<Sweep> autotune_candidates(uint32_t n, int dtype, uint64_t seed) {
  std::mt19937_64 rng(seed);
  std::vector<Sweep> out;
  auto gate = [&](uint32_t k, const std::vector<uint32_t>& qs, std::vector<cd> mat) {
    Gate g;
    g.m = k;
    for (uint32_t j = 0; j < k; ++j) g.q[j] = qs[j];
    g.a = std::move(mat);
    return g;
  };
  // 1q butterflies across the target positions that select kernel variants
  for (uint32_t t : {0u, 1u, 2u, 4u, 6u, 8u, n / 2, n - 1})
    if (t < n) out.push_back(classify_gate(gate(1, {t}, haar(1, rng))));
  // controlled butterflies
  const std::vector<std::pair<uint32_t, uint32_t>> cts = {{0, 1}, {1, 0}, {n - 1, n - 2}, {3, n - 1}, {n - 1, 2}};
  for (auto [c, t] : cts) {
    std::vector<cd> u = haar(1, rng), m(16, cd(0, 0));
    m[0] = m[10] = 1.0;
    m[5] = u[0];
    m[7] = u[1];
    m[13] = u[2];
    m[15] = u[3];
    out.push_back(classify_gate(gate(2, {c, t}, m)));
  }
  // diagonals: CZ-like (identity halves skipped) and general phases
  for (uint32_t k = 1; k <= 6; ++k)
    for (const auto& qs : placements(k, n)) {
      std::uniform_real_distribution<double> ud(0, 6.283185307179586);
      const size_t d = size_t(1) << k;
      std::vector<cd> m(d * d, cd(0, 0));
      for (size_t i = 0; i < d; ++i) m[i * d + i] = std::polar(1.0, ud(rng));
      out.push_back(classify_gate(gate(k, qs, m)));
      if (k == 2) {
        std::vector<cd> cz(16, cd(0, 0));
        cz[0] = cz[5] = cz[10] = 1.0;
        cz[15] = -1.0;
        out.push_back(classify_gate(gate(2, qs, cz)));
      }
    }
  // phase polynomials of 8 / 24 / 60 two-qubit terms
  for (uint32_t nt : {8u, 24u, 60u}) {
    Sweep s;
    s.kind = SK_PHASE;
    std::uniform_int_distribution<uint32_t> uq(0, n - 1);
    std::uniform_real_distribution<double> ud(0, 6.283185307179586);
    for (uint32_t i = 0; i < nt; ++i) {
      PhaseTerm t{};
      t.m = 2;
      t.q[0] = uq(rng);
      do t.q[1] = uq(rng);
      while (t.q[1] == t.q[0]);
      const double a = ud(rng);
      t.ang[0] = t.ang[3] = -0.5 * a;
      t.ang[1] = t.ang[2] = 0.5 * a;
      s.terms.push_back(t);
    }
    s.n_gates = nt;
    out.push_back(s);
  }
  // dense k = 2..6 on CUDA cores, and k = 4..6 on tensor cores (complex64)
  for (uint32_t k = 2; k <= 6; ++k)
    for (const auto& qs : placements(k, n)) {
      Sweep s = classify_gate(gate(k, qs, haar(k, rng)));
      if (s.kind != SK_DENSE) continue;
      out.push_back(s);
      if (dtype == QSVB_C64 && tc_dense_supported(s, n)) {
        Sweep t = s;
        t.kind = SK_DENSE_TC;
        out.push_back(t);
      }
    }
  return out;
}

}  // namespace qsvb

using namespace qsvb;

extern "C" int qsvb_autotune(qsvb_ctx* c, uint32_t n, int dtype, int reps, uint64_t seed, float* features,
                             double* seconds, uint32_t* kinds, size_t cap, size_t* count) {
  try {
    QSVB_REQUIRE(c && count, "null pointer");
    QSVB_REQUIRE(n >= 12 && n <= 32, "autotune qubit count must be 12..32");
    QSVB_REQUIRE(dtype == QSVB_C64 || dtype == QSVB_C128, "dtype must be QSVB_C64 or QSVB_C128");
    QSVB_REQUIRE(reps >= 1 && reps <= 100, "reps must be 1..100");
    const std::vector<Sweep> cands = autotune_candidates(n, dtype, seed);
    *count = cands.size();
    if (!features) return QSVB_OK;
    QSVB_REQUIRE(seconds && kinds && cap >= cands.size(), "output arrays too small");
    QSVB_CK(cudaSetDevice(c->device));
    qsvb_state* st = nullptr;
    int rc = qsvb_state_alloc(c, n, dtype, &st);
    if (rc) return rc;
    struct Free {
      qsvb_ctx* c;
      qsvb_state* s;
      ~Free() { qsvb_state_free(c, s); }
    } guard{c, st};
    rc = qsvb_init_basis(c, st, 0);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    QSVB_CK(cudaEventCreate(&e0));
    QSVB_CK(cudaEventCreate(&e1));
    std::vector<char> host;
    void* dmat = nullptr;
    size_t dcap = 0;
    for (size_t i = 0; i < cands.size(); ++i) {
      const Sweep& s = cands[i];
      const size_t mb = sweep_matrix_bytes(s, dtype);
      if (mb > dcap) {
        if (dmat) QSVB_CK(cudaFree(dmat));
        QSVB_CK(cudaMalloc(&dmat, mb));
        dcap = mb;
      }
      if (mb) {
        host.assign(mb, 0);
        pack_sweep_matrix(s, dtype, host.data());
        QSVB_CK(cudaMemcpy(dmat, host.data(), mb, cudaMemcpyHostToDevice));
      }
      auto run = [&] {
        if (dtype == QSVB_C128)
          launch_sweep<double>(c->env(), static_cast<double*>(st->re), static_cast<double*>(st->im), n, s, dmat);
        else
          launch_sweep<float>(c->env(), static_cast<float*>(st->re), static_cast<float*>(st->im), n, s, dmat);
      };
      run();
      QSVB_CK(cudaEventRecord(e0, c->stream));
      for (int r = 0; r < reps; ++r) run();
      QSVB_CK(cudaEventRecord(e1, c->stream));
      QSVB_CK(cudaEventSynchronize(e1));
      float ms = 0;
      QSVB_CK(cudaEventElapsedTime(&ms, e0, e1));
      seconds[i] = double(ms) * 1e-3 / reps;
      kinds[i] = uint32_t(s.kind);
      sweep_features(s, n, dtype, features + i * kNumFeatures);
    }
    if (dmat) cudaFree(dmat);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int flag = 0;
    QSVB_CK(cudaMemcpy(&flag, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
      QSVB_CK(cudaMemset(c->d_err, 0, sizeof(int)));
      throw Error(QSVB_E_TIMEOUT, "a device-side wait ran out during autotuning");
    }
    return QSVB_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}
