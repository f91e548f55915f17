// Sweep cost model and the learned planner (see cost_model.h).

#include "cost_model.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>
#include <mutex>
#include <unordered_map>

namespace qsvb {

namespace {
std::mutex g_model_mu;
MlpModel g_model;
std::atomic<uint64_t> g_model_generation{0};  // bumped by install_model; keys the prediction memo

// Roofline constants for one B200 (measured copy bandwidth ~6.5 TB/s; sustained fractions).
constexpr double kHbmBytesPerSec = 6.0e12;
constexpr double kFp32FmaFlops = 40.0e12;   // CUDA-core complex GEMM, achieved
constexpr double kFp64FmaFlops = 25.0e12;
constexpr double kTcFlops = 1.2e15;         // bf16 tcgen05, achieved
constexpr double kLaunchSeconds = 2.5e-6;
// tile sweeps: time = factor x (a plain streaming sweep's memory time) + the emitted program's
// arithmetic per amplitude / rate (fitted to 139 measured passes of QFT, brickwork, QAOA, GHZ,
// random and ansatz circuits at 28-30 qubits on one B200: mean |log2 error| 0.18 / 0.16)
constexpr double kTileFp32Flops = 29.5e12;
constexpr double kTileFp64Flops = 15.5e12;
constexpr double kTileMemFactor32 = 1.95;
constexpr double kTileMemFactor64 = 1.80;
// chain and permutation passes (not in the cost model's training records: roofline times an
// overhead factor)
constexpr double kChainOverhead = 1.25;
constexpr double kPermuteOverhead = 1.15;

int lowest_bit(const Sweep& s) {
  uint32_t lo = 64;
  for (uint32_t j = 0; j < s.m; ++j) lo = std::min(lo, s.q[j]);
  if (s.kind == SK_1Q || s.kind == SK_CTRL) lo = s.target;
  return int(lo);
}
}  // namespace

void sweep_features(const Sweep& s, uint32_t n, int dtype, float* f) {
  std::fill(f, f + kNumFeatures, 0.0f);
  const int kind = std::min<int>(s.kind, 6);
  f[kind] = 1.0f;                                    // 0..6 one-hot kind
  f[7] = float(n);
  f[8] = dtype == QSVB_C128 ? 1.0f : 0.0f;
  uint32_t k = s.m;
  if (s.kind == SK_1Q || s.kind == SK_CTRL) k = 1 + s.nctrl;
  if (s.kind == SK_PHASE) k = 0;
  f[9] = float(k);
  f[10] = float(s.nctrl);
  int lo = lowest_bit(s), hi = 0;
  for (uint32_t j = 0; j < s.m; ++j) hi = std::max<int>(hi, int(s.q[j]));
  if (s.kind == SK_1Q || s.kind == SK_CTRL) hi = std::max<int>(hi, int(s.target));
  f[11] = float(std::min(lo, 40));
  f[13] = float(s.terms.size()) / 16.0f;
  if (s.kind == SK_DENSE || s.kind == SK_DENSE_TC) {
    // the dense kernels' tile: gate bits + the (12 - k) lowest other bits; its memory pattern is
    // set by how many runs of consecutive state bits it spans and by which bits are the lowest two
    bool gate[64] = {false}, tile[64] = {false};
    for (uint32_t j = 0; j < s.m; ++j) gate[s.q[j]] = tile[s.q[j]] = true;
    uint32_t ncol = 0;
    for (uint32_t b = 0; b < n && ncol < 12 - s.m; ++b)
      if (!gate[b]) {
        tile[b] = true;
        ++ncol;
      }
    uint32_t runs = 0;
    for (uint32_t b = 0; b < n; ++b) runs += tile[b] && (b == 0 || !tile[b - 1]);
    f[12] = float(runs);
    f[14] = (!gate[0] && !gate[1]) ? 0.0f : (gate[0] && gate[1] ? 1.0f : 2.0f);
  } else {
    f[12] = float(hi);
    uint32_t nlow = 0;
    for (uint32_t j = 0; j < s.m; ++j) nlow += s.q[j] < 7;
    f[14] = float(nlow);
  }
  f[15] = float(std::log2(analytic_sweep_seconds(s, n, dtype)));
}

double analytic_sweep_seconds(const Sweep& s, uint32_t n, int dtype) {
  const double b = dtype == QSVB_C128 ? 16.0 : 8.0;
  const double dim = std::ldexp(1.0, int(n));
  double amps = dim;
  const int sector_bits = dtype == QSVB_C128 ? 2 : 3;  // a 32-byte sector holds 2^bits amplitudes
  uint32_t skip = 0;
  for (uint32_t i = 0; i < s.nctrl; ++i) skip += int(s.ctrl[i]) >= sector_bits;
  if (s.kind == SK_CTRL || s.kind == SK_DIAG) amps = std::ldexp(dim, -int(skip));
  double mem = 2.0 * amps * b / kHbmBytesPerSec;
  double comp = 0.0;
  if (s.kind == SK_DENSE)
    comp = 8.0 * std::ldexp(1.0, int(s.m)) * dim / (dtype == QSVB_C128 ? kFp64FmaFlops : kFp32FmaFlops);
  if (s.kind == SK_DENSE_TC) comp = 3.0 * 8.0 * std::ldexp(1.0, int(s.m)) * dim / kTcFlops;
  if (s.kind == SK_PHASE) comp = double(s.terms.size()) * 4.0 * dim / 30.0e12 + 40.0 * dim / kFp64FmaFlops;
  if (s.kind == SK_TC_CHAIN) {
    // one read and one write of the state; per matrix three bf16 MMAs (1536 flops an amplitude)
    // and its operand traffic through shared memory, overlapped with the memory stream
    const double per_mat = 1536.0 * dim / kTcFlops;
    return std::max(mem, double(s.chain_nmat) * per_mat) * kChainOverhead + kLaunchSeconds;
  }
  if (s.kind == SK_PERMUTE) return mem * kPermuteOverhead + kLaunchSeconds;
  if (s.kind == SK_TILE) {
    // each block loads, updates and stores its tile in turn: memory and arithmetic add up
    const double rate = dtype == QSVB_C128 ? kTileFp64Flops : kTileFp32Flops;
    const double mf = dtype == QSVB_C128 ? kTileMemFactor64 : kTileMemFactor32;
    return mf * mem + s.tile_flops / rate + kLaunchSeconds;
  }
  return std::max(mem, comp) + kLaunchSeconds;
}

const MlpModel& installed_model() { return g_model; }

void install_model(const MlpModel& m) {
  std::lock_guard<std::mutex> lk(g_model_mu);
  g_model = m;
  g_model_generation.fetch_add(1);
}

float mlp_forward_host(const MlpModel& m, const float* feat) {
  const int H = m.hidden;
  constexpr int kStackH = 128;  // widest model the trainer accepts
  float xs[kNumFeatures], h1s[kStackH], h2s[kStackH];
  std::vector<float> h1v, h2v;
  float* x = xs;
  float* h1 = h1s;
  float* h2 = h2s;
  if (H > kStackH) {
    h1v.resize(H);
    h2v.resize(H);
    h1 = h1v.data();
    h2 = h2v.data();
  }
  for (int i = 0; i < kNumFeatures; ++i) x[i] = (feat[i] - m.mean[i]) * m.scale[i];
  for (int j = 0; j < H; ++j) {
    float a = m.b1[j];
    for (int i = 0; i < kNumFeatures; ++i) a += m.w1[j * kNumFeatures + i] * x[i];
    h1[j] = a > 0 ? a : 0;
  }
  for (int j = 0; j < H; ++j) {
    float a = m.b2[j];
    for (int i = 0; i < H; ++i) a += m.w2[j * H + i] * h1[i];
    h2[j] = a > 0 ? a : 0;
  }
  float y = m.b3[0];
  for (int i = 0; i < H; ++i) y += m.w3[i] * h2[i];
  return y * m.y_scale + m.y_mean;
}

namespace {
// The planner predicts the same sweeps many times (the same shapes recur across layers and
// fusion candidates): each thread memoises predictions by feature vector for the installed model.
struct FeatKey {
  float f[kNumFeatures];
  bool operator==(const FeatKey& o) const { return std::memcmp(f, o.f, sizeof(f)) == 0; }
};
struct FeatHash {
  size_t operator()(const FeatKey& k) const {
    uint64_t h = 1469598103934665603ull;
    const unsigned char* p = reinterpret_cast<const unsigned char*>(k.f);
    for (size_t i = 0; i < sizeof(k.f); ++i) h = (h ^ p[i]) * 1099511628211ull;
    return size_t(h);
  }
};

float mlp_forward_host_memo(const MlpModel& m, const float* feat) {
  thread_local std::unordered_map<FeatKey, float, FeatHash> memo;
  thread_local uint64_t memo_gen = ~uint64_t(0);
  const uint64_t gen = g_model_generation.load();
  if (gen != memo_gen || memo.size() > (1u << 16)) {
    memo.clear();
    memo_gen = gen;
  }
  FeatKey k;
  std::memcpy(k.f, feat, sizeof(k.f));
  auto it = memo.find(k);
  if (it != memo.end()) return it->second;
  const float y = mlp_forward_host(m, feat);
  memo.emplace(k, y);
  return y;
}

// Largest state the installed model has seen (its records span 22..30 qubits). A ReLU network
// extrapolates linearly in its inputs, which for larger states put some predictions below the
// memory floor; larger states are predicted as the same sweep on a kModelMaxQubits state times
// the amplitude ratio.
constexpr uint32_t kModelMaxQubits = 30;

// The sweep with d = n - kModelMaxQubits state bits removed: the d highest bits >= 12 that no
// qubit of the sweep uses, the others renumbered below them (low bits, which set the access
// pattern, keep their positions).
Sweep shrink_sweep(const Sweep& s, uint32_t n) {
  const uint32_t d = n - kModelMaxQubits;
  bool used[64] = {false};
  for (uint32_t j = 0; j < s.m; ++j) used[s.q[j]] = true;
  for (uint32_t j = 0; j < s.nctrl; ++j) used[s.ctrl[j]] = true;
  if (s.kind == SK_1Q || s.kind == SK_CTRL) used[s.target] = true;
  bool drop[64] = {false};
  uint32_t dropped = 0;
  for (int b = int(n) - 1; b >= 12 && dropped < d; --b)
    if (!used[b]) drop[b] = true, ++dropped;
  uint32_t to[64];
  for (uint32_t b = 0, below = 0; b < n; ++b) {
    to[b] = b - below;
    below += drop[b];
  }
  Sweep t;
  t.kind = s.kind;
  t.m = s.m;
  t.target = to[s.target];
  t.nctrl = s.nctrl;
  for (uint32_t j = 0; j < 6; ++j) {
    t.q[j] = j < s.m ? to[s.q[j]] : 0;
    t.ctrl[j] = j < s.nctrl ? to[s.ctrl[j]] : 0;
  }
  t.terms.resize(s.terms.size());
  t.n_gates = s.n_gates;
  return t;
}
}  // namespace

double predict_sweep_seconds(const Sweep& s, uint32_t n, int dtype) {
  const MlpModel& m = g_model;
  // the model has not been trained on tile, chain or permutation passes
  if (m.hidden > 0 && s.kind != SK_TILE && s.kind != SK_TC_CHAIN && s.kind != SK_PERMUTE) {
    float f[kNumFeatures];
    if (n > kModelMaxQubits && n - kModelMaxQubits <= 20) {
      sweep_features(shrink_sweep(s, n), kModelMaxQubits, dtype, f);
      return std::ldexp(std::exp2(double(mlp_forward_host_memo(m, f))), int(n - kModelMaxQubits));
    }
    sweep_features(s, n, dtype, f);
    return std::exp2(double(mlp_forward_host_memo(m, f)));
  }
  return analytic_sweep_seconds(s, n, dtype);
}

double predict_plan_seconds(const std::vector<Sweep>& sw, uint32_t n, int dtype) {
  double t = 0;
  for (const Sweep& s : sw) t += predict_sweep_seconds(s, n, dtype);
  return t;
}

void select_engines(std::vector<Sweep>& sw, uint32_t n, const qsvb_plan_opts& o, int dtype) {
  const bool learned = g_model.hidden > 0 && o.planner == QSVB_PLAN_LEARNED;
  for (Sweep& s : sw) {
    if (s.kind != SK_DENSE) continue;
    if (dtype != QSVB_C64 || !tc_dense_supported(s, n) || o.engine == QSVB_ENGINE_CUDA_CORE) continue;
    if (o.engine == QSVB_ENGINE_TENSOR_CORE) {
      s.kind = SK_DENSE_TC;
    } else if (learned) {  // auto + trained model: the cheaper engine by prediction
      Sweep t = s;
      t.kind = SK_DENSE_TC;
      if (predict_sweep_seconds(t, n, dtype) < predict_sweep_seconds(s, n, dtype)) s.kind = SK_DENSE_TC;
    } else if (s.m >= 5) {  // auto without a model: tensor cores once CUDA cores turn compute-bound
      s.kind = SK_DENSE_TC;
    }
  }
}

std::vector<Gate> learned_fuse(const std::vector<Gate>& seg, uint32_t n, const qsvb_plan_opts& o, int dtype) {
  const uint32_t cap = std::max<uint32_t>(1, o.max_fused_qubits);
  // every (strategy, width) candidate is grouped, classified and costed independently (on long
  // segments on separate host threads), without composing the matrices of groups whose sweep
  // kind does not depend on them; only the chosen candidate is composed
  auto candidate = [&](int strategy, uint32_t k) {
    const std::vector<Gate> cand = strategy == 0 ? fuse_greedy_public(seg, k, true) : fuse_window_public(seg, k, true);
    std::vector<Sweep> sw;
    sw.reserve(cand.size());
    for (const Gate& g : cand) {
      Sweep s;
      if (g.a.empty()) {  // uncomposed group of >= 3 qubits: a dense sweep on its sorted qubits
        s.kind = SK_DENSE;
        s.m = g.m;
        for (uint32_t j = 0; j < g.m; ++j) s.q[j] = g.q[j];
        std::sort(s.q, s.q + g.m);
        s.n_gates = 1;
      } else {
        s = classify_gate(g);
      }
      if (s.kind != SK_NONE) sw.push_back(std::move(s));
    }
    select_engines(sw, n, o, dtype);
    return predict_plan_seconds(sw, n, dtype);
  };
  const size_t ncand = 2 * size_t(cap);
  std::vector<double> secs(ncand, 1e300);
  parallel_ranges(ncand, seg.size() >= 64 ? 1 : SIZE_MAX, [&](size_t lo, size_t hi) {
    for (size_t c = lo; c < hi; ++c) secs[c] = candidate(int(c / cap), uint32_t(c % cap) + 1);
  });
  size_t best = 0;
  for (size_t c = 1; c < ncand; ++c)
    if (secs[c] < secs[best]) best = c;  // ties keep the earlier (greedy, narrower) candidate
  const uint32_t k = uint32_t(best % cap) + 1;
  return best / cap == 0 ? fuse_greedy_public(seg, k) : fuse_window_public(seg, k);
}

}  // namespace qsvb
