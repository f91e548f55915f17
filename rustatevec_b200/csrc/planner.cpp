// Host planner: input gates -> fused gates -> classified sweeps.
//
// * GREEDY follows qsv's fuse (crates/qsv-core/src/fusion.rs:39-100): consecutive-only grouping
//   while the union of qubits stays <= max; single-gate groups pass through unchanged, larger
//   groups are composed onto their sorted qubit set (fusion.rs:102-140). Composition here is FP64
//   whatever the state precision.
// * WINDOW grows each group past gates it cannot absorb, as long as every absorbed gate acts on
//   qubits disjoint from all gates it jumps over (such gates commute, so the result is exact).
// * LEARNED picks, per circuit, the cheapest of the candidate plans under the cost model
//   (cost_model.cpp); GREEDY at the requested width is always among the candidates.
// * Runs of >= 3 consecutive diagonal gates of <= 2 qubits whose qubit union exceeds the fusion
//   width become one phase-polynomial sweep (WINDOW and LEARNED).
//
// classify_gate mirrors the dispatch of qsv's CudaBackend::apply / CpuBackend::apply
// (crates/qsv-cuda/src/lib.rs:121-200, crates/qsv-core/src/backend/cpu.rs:281-290): diagonal ->
// diagonal sweep, one qubit -> butterfly, else dense, with one addition: a gate that is the
// identity whenever some of its qubits are 0 and a 2x2 on the one remaining qubit is a controlled
// butterfly that only visits the control=1 subspace.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <numeric>
#include <thread>

#include "cost_model.h"
#include "qsvb_internal.h"

namespace qsvb {

thread_local uint32_t g_plan_threads = 0;

qsvb_plan_opts default_opts() {
  qsvb_plan_opts o{};
  o.planner = QSVB_PLAN_GREEDY;
  o.max_fused_qubits = 4;
  o.engine = QSVB_ENGINE_AUTO;
  o.use_graph = 1;
  return o;
}

void validate_circuit(const qsvb_circuit* c) {
  QSVB_REQUIRE(c != nullptr, "null circuit");
  QSVB_REQUIRE(c->n_qubits >= 1 && c->n_qubits <= QSVB_MAX_QUBITS, "circuit qubit count out of range");
  QSVB_REQUIRE(c->n_gates == 0 || c->gates != nullptr, "null gate array");
  for (size_t i = 0; i < c->n_gates; ++i) {
    const qsvb_gate& g = c->gates[i];
    QSVB_REQUIRE(g.n_qubits >= 1 && g.n_qubits <= QSVB_MAX_GATE_QUBITS,
                 "gate " + std::to_string(i) + ": arity must be 1..6");
    QSVB_REQUIRE(g.n_qubits <= c->n_qubits, "gate " + std::to_string(i) + ": more qubits than the register");
    QSVB_REQUIRE(g.matrix != nullptr, "gate " + std::to_string(i) + ": null matrix");
    for (uint32_t j = 0; j < g.n_qubits; ++j) {
      QSVB_REQUIRE(g.qubits[j] < c->n_qubits, "gate " + std::to_string(i) + ": qubit " +
                                                  std::to_string(g.qubits[j]) + " out of range for " +
                                                  std::to_string(c->n_qubits) + " qubits");
      for (uint32_t k = j + 1; k < g.n_qubits; ++k)
        QSVB_REQUIRE(g.qubits[j] != g.qubits[k], "gate " + std::to_string(i) + ": repeated qubit in gate");
    }
  }
}

std::vector<Gate> gates_from_circuit(const qsvb_circuit* c) {
  std::vector<Gate> out(c->n_gates);
  for (size_t i = 0; i < c->n_gates; ++i) {
    const qsvb_gate& g = c->gates[i];
    Gate& o = out[i];
    o.m = g.n_qubits;
    for (uint32_t j = 0; j < o.m; ++j) o.q[j] = g.qubits[j];
    const size_t d = size_t(1) << o.m;
    o.a.resize(d * d);
    for (size_t k = 0; k < d * d; ++k) o.a[k] = cd(g.matrix[2 * k], g.matrix[2 * k + 1]);
  }
  return out;
}

namespace {

uint64_t qmask(const Gate& g) {
  uint64_t m = 0;
  for (uint32_t j = 0; j < g.m; ++j) m |= 1ull << g.q[j];
  return m;
}

bool is_diag(const Gate& g) {
  const size_t d = size_t(1) << g.m;
  for (size_t r = 0; r < d; ++r)
    for (size_t c = 0; c < d; ++c)
      if (r != c && g.a[r * d + c] != cd(0.0, 0.0)) return false;
  return true;
}

// Compose `ops` (applied in order) onto the sorted qubit list `q` in FP64: new = E(g) * mat, the
// embedding qsv's build_fused uses (fusion.rs:102-140). Each gate updates, in place, the 2^m rows
// it mixes (rows whose indices differ only in the gate's bits), with real and imaginary parts in
// separate arrays; every product is summed in gate-column order from zero, skipping zero entries.
// A new row is accumulated 8 columns at a time in registers over all of the gate's nonzero
// entries of that row (the same sums in the same order as one pass per entry, with a third of the
// loads and stores). An AVX2 clone is chosen at load time where the host has it (no FMA: the
// same roundings as the default SSE2 clone).
__attribute__((target_clones("avx2", "default")))
Gate compose(const std::vector<uint32_t>& q, const std::vector<const Gate*>& ops) {
  const size_t m = q.size(), dim = size_t(1) << m;
  std::vector<double> re(dim * dim, 0.0), im(dim * dim, 0.0);  // row-major
  for (size_t i = 0; i < dim; ++i) re[i * dim + i] = 1.0;
  std::vector<double> ore, oim;  // the old values of the rows one gate block mixes
  std::vector<double> ger, gei;  // per gate row: the nonzero entries, in column order
  std::vector<uint8_t> gks;      // ... and their columns
  for (const Gate* g : ops) {
    const size_t nsub = size_t(1) << g->m;
    size_t off[64], gmask = 0, nnz[64];
    uint32_t local[6];
    for (uint32_t j = 0; j < g->m; ++j) {
      local[j] = uint32_t(std::find(q.begin(), q.end(), g->q[j]) - q.begin());
      gmask |= size_t(1) << local[j];
    }
    for (size_t ks = 0; ks < nsub; ++ks) {
      size_t o = 0;
      for (uint32_t j = 0; j < g->m; ++j) o |= ((ks >> j) & 1u) << local[j];
      off[ks] = o;
    }
    ger.resize(nsub * nsub);
    gei.resize(nsub * nsub);
    gks.resize(nsub * nsub);
    for (size_t rs = 0; rs < nsub; ++rs) {
      nnz[rs] = 0;
      for (size_t ks = 0; ks < nsub; ++ks) {
        const cd e = g->a[rs * nsub + ks];
        if (e == cd(0, 0)) continue;
        ger[rs * nsub + nnz[rs]] = e.real();
        gei[rs * nsub + nnz[rs]] = e.imag();
        gks[rs * nsub + nnz[rs]++] = uint8_t(ks);
      }
    }
    ore.resize(nsub * dim);
    oim.resize(nsub * dim);
    for (size_t b = 0; b < dim; ++b) {
      if (b & gmask) continue;
      for (size_t ks = 0; ks < nsub; ++ks) {
        std::copy_n(&re[(b | off[ks]) * dim], dim, &ore[ks * dim]);
        std::copy_n(&im[(b | off[ks]) * dim], dim, &oim[ks * dim]);
      }
      for (size_t rs = 0; rs < nsub; ++rs) {
        double* __restrict__ dr = &re[(b | off[rs]) * dim];
        double* __restrict__ di = &im[(b | off[rs]) * dim];
        const double* er = &ger[rs * nsub];
        const double* ei = &gei[rs * nsub];
        const uint8_t* kk = &gks[rs * nsub];
        if (dim >= 8) {
          for (size_t c0 = 0; c0 < dim; c0 += 8) {
            double ar[8] = {}, ai[8] = {};
            for (size_t t = 0; t < nnz[rs]; ++t) {
              const double* __restrict__ sr = &ore[kk[t] * dim + c0];
              const double* __restrict__ si = &oim[kk[t] * dim + c0];
              const double xr = er[t], xi = ei[t];
              for (int j = 0; j < 8; ++j) {
                ar[j] += xr * sr[j] - xi * si[j];
                ai[j] += xr * si[j] + xi * sr[j];
              }
            }
            for (int j = 0; j < 8; ++j) {
              dr[c0 + j] = ar[j];
              di[c0 + j] = ai[j];
            }
          }
        } else {
          for (size_t c = 0; c < dim; ++c) {
            double ar = 0.0, ai = 0.0;
            for (size_t t = 0; t < nnz[rs]; ++t) {
              ar += er[t] * ore[kk[t] * dim + c] - ei[t] * oim[kk[t] * dim + c];
              ai += er[t] * oim[kk[t] * dim + c] + ei[t] * ore[kk[t] * dim + c];
            }
            dr[c] = ar;
            di[c] = ai;
          }
        }
      }
    }
  }
  Gate out;
  out.m = uint32_t(m);
  for (size_t j = 0; j < m; ++j) out.q[j] = q[j];
  out.a.resize(dim * dim);
  for (size_t i = 0; i < dim * dim; ++i) out.a[i] = cd(re[i], im[i]);
  return out;
}

// A group of diagonal gates composed as the product of their diagonals (O(2^m) per gate), kept as
// the diagonal alone (candidate costing only needs its classification).
Gate compose_diag(const std::vector<uint32_t>& q, const std::vector<const Gate*>& ops) {
  const size_t m = q.size(), dim = size_t(1) << m;
  std::vector<cd> d(dim, cd(1, 0));
  for (const Gate* g : ops) {
    uint32_t local[6];
    for (uint32_t j = 0; j < g->m; ++j)
      local[j] = uint32_t(std::find(q.begin(), q.end(), g->q[j]) - q.begin());
    const size_t gd = size_t(1) << g->m;
    for (size_t r = 0; r < dim; ++r) {
      size_t rs = 0;
      for (uint32_t j = 0; j < g->m; ++j) rs |= ((r >> local[j]) & 1u) << j;
      d[r] = g->a[rs * gd + rs] * d[r];
    }
  }
  Gate out;
  out.m = uint32_t(m);
  for (size_t j = 0; j < m; ++j) out.q[j] = q[j];
  out.a = std::move(d);
  out.diag_only = true;
  return out;
}

// Emits one fused group. With `cost_only` (candidate costing in the learned planner) a group of
// three or more qubits that holds a non-diagonal gate becomes a placeholder with no matrix (it
// classifies as a dense sweep, whose cost does not depend on the entries); groups whose kind the
// entries decide (diagonal, or at most two qubits) are still composed.
Gate make_group(const std::vector<const Gate*>& grp, bool cost_only) {
  if (grp.size() == 1) return *grp[0];
  uint64_t mask = 0;
  bool all_diag = true;
  for (const Gate* g : grp) {
    mask |= qmask(*g);
    all_diag = all_diag && is_diag(*g);
  }
  std::vector<uint32_t> q;
  for (uint32_t b = 0; b < 64; ++b)
    if ((mask >> b) & 1) q.push_back(b);
  if (cost_only && all_diag) return compose_diag(q, grp);
  if (cost_only && q.size() > 2) {
    Gate ph;
    ph.m = uint32_t(q.size());
    for (size_t j = 0; j < q.size(); ++j) ph.q[j] = q[j];
    return ph;
  }
  return compose(q, grp);
}

// The fused gates of a grouping, in order. Full compositions of many groups run on host threads
// (each group is independent; the result does not depend on the split).
std::vector<Gate> emit_groups(const std::vector<std::vector<const Gate*>>& groups, bool cost_only) {
  std::vector<Gate> out(groups.size());
  auto range = [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) out[i] = make_group(groups[i], cost_only);
  };
  parallel_ranges(groups.size(), cost_only ? SIZE_MAX : 32, range);
  return out;
}

// fusion.rs:39-77 — consecutive-only greedy.
std::vector<Gate> fuse_greedy(const std::vector<Gate>& in, uint32_t maxq, bool cost_only = false) {
  maxq = std::max<uint32_t>(maxq, 1);
  std::vector<std::vector<const Gate*>> groups;
  std::vector<const Gate*> grp;
  std::vector<uint32_t> gq;  // insertion order, as the reference keeps it
  auto close = [&] {
    if (!grp.empty()) groups.push_back(grp);
    grp.clear();
  };
  for (const Gate& g : in) {
    if (g.m > maxq) {
      close();
      gq.clear();
      groups.push_back({&g});
      continue;
    }
    std::vector<uint32_t> uni = gq;
    for (uint32_t j = 0; j < g.m; ++j)
      if (std::find(uni.begin(), uni.end(), g.q[j]) == uni.end()) uni.push_back(g.q[j]);
    if (grp.empty()) {
      gq.assign(g.q, g.q + g.m);
      grp.push_back(&g);
    } else if (uni.size() <= maxq) {
      gq = uni;
      grp.push_back(&g);
    } else {
      close();
      gq.assign(g.q, g.q + g.m);
      grp.push_back(&g);
    }
  }
  close();
  return emit_groups(groups, cost_only);
}

// Commutation-aware window fusion: a later gate may join the open group when its qubits are
// disjoint from every not-yet-emitted gate it would jump over.
std::vector<Gate> fuse_window(const std::vector<Gate>& in, uint32_t maxq, bool cost_only = false,
                              size_t lookahead = 1024) {
  maxq = std::max<uint32_t>(maxq, 1);
  std::vector<char> done(in.size(), 0);
  std::vector<std::vector<const Gate*>> groups;
  size_t first = 0;
  std::vector<const Gate*> grp;
  while (true) {
    while (first < in.size() && done[first]) ++first;
    if (first == in.size()) break;
    done[first] = 1;
    const Gate& g0 = in[first];
    if (g0.m > maxq) {
      groups.push_back({&g0});
      continue;
    }
    grp.assign(1, &g0);
    uint64_t gmask = qmask(g0), blocked = 0;
    size_t scanned = 0;
    for (size_t i = first + 1; i < in.size() && scanned < lookahead; ++i) {
      if (done[i]) continue;
      ++scanned;
      const uint64_t m = qmask(in[i]);
      if ((m & blocked) == 0 && uint32_t(__builtin_popcountll(gmask | m)) <= maxq) {
        grp.push_back(&in[i]);
        done[i] = 1;
        gmask |= m;
      } else {
        blocked |= m;
        // nothing can join once every qubit of a full group is blocked
        if (uint32_t(__builtin_popcountll(gmask)) == maxq && (gmask & ~blocked) == 0) break;
      }
    }
    groups.push_back(grp);
  }
  return emit_groups(groups, cost_only);
}

bool phase_representable(const Gate& g) {
  if (g.m > 2 || !is_diag(g)) return false;
  const size_t d = size_t(1) << g.m;
  for (size_t i = 0; i < d; ++i)
    if (std::abs(std::abs(g.a[i * d + i]) - 1.0) > 1e-12) return false;
  return true;
}

}  // namespace

Gate compose_gates(const std::vector<uint32_t>& q, const std::vector<const Gate*>& ops) { return compose(q, ops); }
uint64_t gate_mask(const Gate& g) { return qmask(g); }

std::vector<Gate> fuse_greedy_public(const std::vector<Gate>& in, uint32_t maxq, bool cost_only) {
  return fuse_greedy(in, maxq, cost_only);
}
std::vector<Gate> fuse_window_public(const std::vector<Gate>& in, uint32_t maxq, bool cost_only) {
  return fuse_window(in, maxq, cost_only);
}

std::vector<Gate> fuse_gates(const std::vector<Gate>& in, uint32_t n, const qsvb_plan_opts& o, int dtype) {
  (void)n;
  (void)dtype;
  switch (o.planner) {
    case QSVB_PLAN_AS_GIVEN: return in;
    case QSVB_PLAN_GREEDY: return fuse_greedy(in, o.max_fused_qubits);
    case QSVB_PLAN_WINDOW: return fuse_window(in, o.max_fused_qubits);
    default: return fuse_window(in, o.max_fused_qubits);
  }
}

Sweep classify_gate(const Gate& g) {
  Sweep s;
  s.m = g.m;
  for (uint32_t j = 0; j < g.m; ++j) s.q[j] = g.q[j];
  s.n_gates = 1;
  const size_t d = size_t(1) << g.m;
  auto at = [&](size_t r, size_t c) { return g.a[r * d + c]; };
  if (g.diag_only || is_diag(g)) {
    auto dg = [&](size_t i) { return g.diag_only ? g.a[i] : at(i, i); };
    bool ident = true;
    for (size_t i = 0; i < d; ++i) ident = ident && dg(i) == cd(1, 0);
    if (ident) {
      s.kind = SK_NONE;
      return s;
    }
    s.kind = SK_DIAG;
    s.mat.resize(d);
    for (size_t i = 0; i < d; ++i) s.mat[i] = dg(i);
    for (uint32_t j = 0; j < g.m; ++j) {  // qubit j is skippable when its 0-half is all ones
      bool ok = true;
      for (size_t i = 0; i < d && ok; ++i)
        if (((i >> j) & 1) == 0 && dg(i) != cd(1, 0)) ok = false;
      if (ok) s.ctrl[s.nctrl++] = g.q[j];
    }
    return s;
  }
  if (g.m == 1) {
    s.kind = SK_1Q;
    s.target = g.q[0];
    s.mat = {at(0, 0), at(0, 1), at(1, 0), at(1, 1)};
    return s;
  }
  // control detection: qubit j is a control when the gate is the identity on its 0-half and
  // never mixes its 0- and 1-halves
  uint32_t ctrl_local = 0;
  for (uint32_t j = 0; j < g.m; ++j) {
    bool ok = true;
    for (size_t r = 0; r < d && ok; ++r)
      for (size_t c = 0; c < d && ok; ++c) {
        const size_t rb = (r >> j) & 1, cb = (c >> j) & 1;
        if (rb != cb) ok = at(r, c) == cd(0, 0);
        else if (rb == 0) ok = at(r, c) == (r == c ? cd(1, 0) : cd(0, 0));
      }
    if (ok) ctrl_local |= 1u << j;
  }
  if (__builtin_popcount(ctrl_local) == int(g.m) - 1) {
    uint32_t tl = 0;
    while ((ctrl_local >> tl) & 1) ++tl;
    s.kind = SK_CTRL;
    s.target = g.q[tl];
    for (uint32_t j = 0; j < g.m; ++j)
      if ((ctrl_local >> j) & 1) s.ctrl[s.nctrl++] = g.q[j];
    const size_t r0 = ctrl_local, r1 = ctrl_local | (size_t(1) << tl);
    s.mat = {at(r0, r0), at(r0, r1), at(r1, r0), at(r1, r1)};
    return s;
  }
  // dense: canonical ascending qubit order (bit i of the index <-> i-th smallest qubit), so the
  // kernels can rely on the gate's lowest qubits being the low bits of the sub-index
  s.kind = SK_DENSE;
  uint32_t order[6];
  for (uint32_t i = 0; i < g.m; ++i) order[i] = i;
  std::sort(order, order + g.m, [&](uint32_t a, uint32_t b) { return g.q[a] < g.q[b]; });
  for (uint32_t i = 0; i < g.m; ++i) s.q[i] = g.q[order[i]];
  size_t remap[64];  // sorted-order index -> gate-order index
  for (size_t sidx = 0; sidx < d; ++sidx) {
    size_t o = 0;
    for (uint32_t i = 0; i < g.m; ++i) o |= ((sidx >> i) & 1u) << order[i];
    remap[sidx] = o;
  }
  s.mat.resize(d * d);
  for (size_t r = 0; r < d; ++r)
    for (size_t c = 0; c < d; ++c) s.mat[r * d + c] = at(remap[r], remap[c]);
  return s;
}

namespace {
enum TileMode { TILE_NO = 0, TILE_ALWAYS = 1, TILE_CHOOSE = 2 };
std::vector<Sweep> plan_with(const std::vector<Gate>& in, uint32_t n, const qsvb_plan_opts& o, int dtype,
                             bool phase_runs, TileMode tile);
}

std::vector<Sweep> plan_sweeps(const std::vector<Gate>& in, uint32_t n, const qsvb_plan_opts& o0, int dtype) {
  qsvb_plan_opts o = o0;
  if (o.max_fused_qubits == 0) o.max_fused_qubits = 1;
  o.max_fused_qubits = std::min<uint32_t>(o.max_fused_qubits, std::min<uint32_t>(QSVB_MAX_GATE_QUBITS, n));
  // tile passes absorb diagonal runs themselves (per-tile phases outside the local set)
  if (o.planner == QSVB_PLAN_TILE) return plan_with(in, n, o, dtype, false, TILE_ALWAYS);
  const bool chain_ok = dtype == QSVB_C64 && n >= 12 && o.engine != QSVB_ENGINE_CUDA_CORE;
  if (o.planner == QSVB_PLAN_CHAIN) {
    if (!chain_ok) {  // chain passes need a complex64 state of >= 12 qubits and the tensor cores
      qsvb_plan_opts w = o;
      w.planner = QSVB_PLAN_WINDOW;
      return plan_with(in, n, w, dtype, false, TILE_NO);
    }
    if (o.chain_max_matrices != 0) return plan_chain(in, n, o.chain_max_matrices);
    std::vector<Sweep> best;
    double best_t = 1e300;
    for (uint32_t m = 1; m <= uint32_t(kChainMaxMats); ++m) {
      std::vector<Sweep> cand = plan_chain(in, n, m);
      const double t = predict_plan_seconds(cand, n, dtype);
      if (t < best_t) {
        best_t = t;
        best = std::move(cand);
      }
    }
    return best;
  }
  if (o.planner != QSVB_PLAN_LEARNED) return plan_with(in, n, o, dtype, false, TILE_NO);
  // learned: merging long diagonal runs into phase-polynomial sweeps, and running gate runs as
  // tile passes, are candidate choices weighed by predicted time
  // the candidates are independent: plan them on separate host threads, each with its share of
  // the host's threads for its own parallel loops
  const bool with_chain = chain_ok && n >= 14;
  const size_t ncand = 4 + (with_chain ? size_t(kChainMaxMats) - 1 : 0);
  const uint32_t share = uint32_t(std::max<size_t>(1, plan_thread_budget() / ncand));
  std::vector<std::future<std::vector<Sweep>>> fut;
  for (int c = 0; c < 4; ++c)
    fut.push_back(std::async(std::launch::async, [&, c] {
      g_plan_threads = share;
      return plan_with(in, n, o, dtype, (c & 1) == 0, c < 2 ? TILE_NO : TILE_CHOOSE);
    }));
  // chain passes (complex64 on the tensor cores, states of >= 14 qubits) at 2 and 3 matrices a pass
  if (with_chain)
    for (uint32_t m = 2; m <= uint32_t(kChainMaxMats); ++m)
      fut.push_back(std::async(std::launch::async, [&, m] {
        g_plan_threads = share;
        return plan_chain(in, n, m);
      }));
  std::vector<Sweep> best;
  double best_t = 1e300;
  for (size_t c = 0; c < fut.size(); ++c) {
    std::vector<Sweep> cand = fut[c].get();
    const double t = predict_plan_seconds(cand, n, dtype);
    if (t < best_t) {
      best_t = t;
      best = std::move(cand);
    }
  }
  return best;
}

namespace {
// Fused sweeps for a run of gates (the planner's fusion, then classification).
std::vector<Sweep> fused_sweeps(const std::vector<Gate>& seg, uint32_t n, const qsvb_plan_opts& o, int dtype) {
  std::vector<Sweep> out;
  if (seg.empty()) return out;
  std::vector<Gate> fused;
  if (o.planner == QSVB_PLAN_LEARNED) {
    fused = learned_fuse(seg, n, o, dtype);
  } else if (o.planner == QSVB_PLAN_TILE) {
    fused = fuse_greedy(seg, o.max_fused_qubits);
  } else {
    fused = fuse_gates(seg, n, o, dtype);
  }
  for (const Gate& g : fused) {
    Sweep s = classify_gate(g);
    if (s.kind == SK_NONE) continue;
    out.push_back(std::move(s));
  }
  return out;
}

// Tile passes over a run of gates. Each pass takes a local set S (qubits 0..4 plus the qubits of
// the first pending non-diagonal gates, up to the tile width) and every pending 1- or 2-qubit gate
// inside S, or diagonal, that commutes past the pending gates it skips (disjoint qubits, or both
// diagonal); wider gates end the run and become fused sweeps. TILE_CHOOSE keeps a pass as a tile sweep only when it is
// predicted faster than the fused sweeps of the same gates.
void tile_segment(const std::vector<Gate>& seg, uint32_t n, const qsvb_plan_opts& o, int dtype, TileMode mode,
                  std::vector<Sweep>& out) {
  const uint32_t L = tile_local_bits(dtype, n);
  auto append = [&](std::vector<Sweep>&& v) {
    for (Sweep& s : v) out.push_back(std::move(s));
  };
  if (L == 0) {
    append(fused_sweeps(seg, n, o, dtype));
    return;
  }
  std::vector<Gate> pend;
  std::vector<Sweep> passes;  // the tile passes of one run of gates, in order
  auto flush = [&] {
    std::vector<char> done(pend.size(), 0);
    size_t first = 0;
    while (true) {
      while (first < pend.size() && done[first]) ++first;
      if (first == pend.size()) break;
      // diagonal gates never force a qubit into the tile (outside it their entries are fixed per
      // tile), so the local set follows the pending non-diagonal gates
      uint64_t S = 31;
      for (size_t i = first; i < pend.size() && uint32_t(__builtin_popcountll(S)) < L; ++i) {
        if (done[i] || is_diag(pend[i])) continue;
        const uint64_t m = qmask(pend[i]);
        if (uint32_t(__builtin_popcountll(S | m)) <= L) S |= m;
      }
      for (uint32_t b = 5; b < n && uint32_t(__builtin_popcountll(S)) < L; ++b) S |= 1ull << b;
      uint64_t blocked = 0, dblocked = 0;
      Sweep t;
      t.kind = SK_TILE;
      t.tile_mask = S;
      for (size_t i = first; i < pend.size(); ++i) {
        if (done[i]) continue;
        const uint64_t m = qmask(pend[i]);
        const bool diag = is_diag(pend[i]);
        if ((diag || (m & ~S) == 0) && (m & blocked) == 0 && (diag || (m & dblocked) == 0)) {
          done[i] = 1;
          t.tile_gates.push_back(pend[i]);
        } else if (diag) {
          dblocked |= m;
        } else {
          blocked |= m;
        }
      }
      passes.push_back(std::move(t));
    }
    pend.clear();
    // A pass's gates do not depend on how earlier passes were run, so each pass is prepared (and,
    // with TILE_CHOOSE, weighed against the fused sweeps of its gates) on its own: long runs of
    // passes spread over host threads, and the results are appended in pass order.
    std::vector<std::vector<Sweep>> res(passes.size());
    auto work = [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; ++i) {
        Sweep& t = passes[i];
        if (mode == TILE_CHOOSE) {
          std::vector<Sweep> alt = fused_sweeps(t.tile_gates, n, o, dtype);
          select_engines(alt, n, o, dtype);
          tile_prepare(t, n, dtype);
          if (predict_plan_seconds(alt, n, dtype) <= predict_sweep_seconds(t, n, dtype)) {
            res[i] = std::move(alt);
            continue;
          }
        } else {
          tile_prepare(t, n, dtype);
        }
        res[i].push_back(std::move(t));
      }
    };
    parallel_ranges(passes.size(), 4, work);
    passes.clear();
    for (auto& r : res) append(std::move(r));
  };
  for (const Gate& g : seg) {
    if (g.m <= 2) {
      pend.push_back(g);
    } else {
      flush();
      append(fused_sweeps(std::vector<Gate>{g}, n, o, dtype));
    }
  }
  flush();
}

std::vector<Sweep> plan_with(const std::vector<Gate>& in, uint32_t n, const qsvb_plan_opts& o, int dtype,
                             bool phase_runs, TileMode tile) {

  // split into segments: phase-polynomial runs vs ordinary gates. Segments are planned
  // independently (on several host threads when there are many) and concatenated in order.
  struct Part {
    std::vector<Gate> seg;  // gates to fuse / tile, or
    Sweep phase;            // a ready phase-polynomial sweep (seg empty)
  };
  std::vector<Part> parts;
  auto run_segment = [&](const std::vector<Gate>& seg) {
    if (seg.empty()) return;
    parts.emplace_back();
    parts.back().seg = seg;
  };
  std::vector<Gate> seg;
  size_t i = 0;
  while (i < in.size()) {
    if (phase_runs && phase_representable(in[i])) {
      size_t j = i;
      uint64_t mask = 0;
      while (j < in.size() && phase_representable(in[j])) mask |= qmask(in[j++]);
      if (j - i >= 3 && uint32_t(__builtin_popcountll(mask)) > o.max_fused_qubits) {
        run_segment(seg);
        seg.clear();
        Sweep s;
        s.kind = SK_PHASE;
        s.n_gates = j - i;
        for (size_t k = i; k < j; ++k) {
          const Gate& g = in[k];
          PhaseTerm t{};
          t.m = g.m;
          for (uint32_t a = 0; a < g.m; ++a) t.q[a] = g.q[a];
          const size_t d = size_t(1) << g.m;
          for (size_t e = 0; e < 4; ++e) t.ang[e] = e < d ? std::arg(g.a[e * d + e]) : 0.0;
          s.terms.push_back(t);
        }
        parts.emplace_back();
        parts.back().phase = std::move(s);
        i = j;
        continue;
      }
      for (size_t k = i; k < j; ++k) seg.push_back(in[k]);
      i = j;
      continue;
    }
    seg.push_back(in[i++]);
  }
  run_segment(seg);

  std::vector<std::vector<Sweep>> res(parts.size());
  auto work = [&](size_t lo, size_t hi) {
    for (size_t k = lo; k < hi; ++k) {
      if (parts[k].seg.empty()) {
        res[k].push_back(std::move(parts[k].phase));
      } else if (tile != TILE_NO) {
        tile_segment(parts[k].seg, n, o, dtype, tile, res[k]);
      } else {
        res[k] = fused_sweeps(parts[k].seg, n, o, dtype);
      }
    }
  };
  parallel_ranges(parts.size(), 4, work);
  std::vector<Sweep> out;
  for (auto& r : res)
    for (Sweep& s : r) out.push_back(std::move(s));
  select_engines(out, n, o, dtype);
  return out;
}
}  // namespace

void sweep_costs(const std::vector<Sweep>& sw, uint32_t n, int dtype, qsvb_plan_stats* st) {
  const double b = dtype == QSVB_C128 ? 16.0 : 8.0;
  const double dim = std::ldexp(1.0, int(n));
  st->n_sweeps = sw.size();
  for (auto& k : st->n_sweeps_by_kind) k = 0;
  st->algorithmic_bytes = st->full_sweep_bytes = st->flops = 0;
  for (const Sweep& s : sw) {
    int kind = s.kind;
    st->n_sweeps_by_kind[kind < kNumSweepKinds ? kind : 7]++;
    double amps = dim;
    if (s.kind == SK_CTRL) amps = std::ldexp(dim, -int(s.nctrl));
    if (s.kind == SK_DIAG) amps = std::ldexp(dim, -int(s.nctrl));
    st->algorithmic_bytes += 2.0 * amps * b;
    st->full_sweep_bytes += 2.0 * dim * b;
    if (s.kind == SK_DENSE || s.kind == SK_DENSE_TC) st->flops += 8.0 * std::ldexp(1.0, int(s.m)) * dim;
    if (s.kind == SK_TILE) st->flops += s.tile_flops;
    if (s.kind == SK_TC_CHAIN) st->flops += double(s.chain_nmat) * 8.0 * 64.0 * dim;
  }
  st->predicted_seconds = predict_plan_seconds(sw, n, dtype);
  st->measured_seconds = 0.0;
}

}  // namespace qsvb
