// The learned part of the planner: a small MLP cost model (features of a sweep -> log2 seconds),
// trained on the GPU by the kernels below on the autotuner's timing records.
//
// Model: x = (f - mean) * scale; h1 = relu(W1 x + b1); h2 = relu(W2 h1 + b2); y = w3 . h2 + b3;
// prediction = y * y_scale + y_mean (log2 seconds). Loss = mean over samples of (y - t)^2 with
// t = (log2 seconds - y_mean) / y_scale. Parameters are one flat float vector:
//   [W1 (H x F) | b1 (H) | W2 (H x H) | b2 (H) | w3 (H) | b3 (1)]
// Training is full-batch Adam. The backward pass writes one gradient row per sample and a second
// kernel sums the rows in a fixed order, so a training run is deterministic.

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "cost_model.h"
#include "qsvb_internal.h"

namespace qsvb {
namespace {

constexpr int F = kNumFeatures;
constexpr int kMaxHidden = 128;

__host__ __device__ inline size_t n_params(int H) { return size_t(H) * F + H + size_t(H) * H + H + H + 1; }

struct Offsets {
  size_t w1, b1, w2, b2, w3, b3;
};
__host__ __device__ inline Offsets offsets(int H) {
  Offsets o;
  o.w1 = 0;
  o.b1 = o.w1 + size_t(H) * F;
  o.w2 = o.b1 + H;
  o.b2 = o.w2 + size_t(H) * H;
  o.w3 = o.b2 + H;
  o.b3 = o.w3 + H;
  return o;
}

// One thread per sample: forward pass, loss term, and that sample's gradient row.
__global__ void k_mlp_fwd_bwd(const float* __restrict__ P, int H, const float* __restrict__ X,
                              const float* __restrict__ T, int n, float* __restrict__ G, float* __restrict__ L) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Offsets o = offsets(H);
  const float* x = X + size_t(i) * F;
  float h1[kMaxHidden], h2[kMaxHidden], d2[kMaxHidden];
  for (int j = 0; j < H; ++j) {
    float a = P[o.b1 + j];
    for (int f = 0; f < F; ++f) a = fmaf(P[o.w1 + size_t(j) * F + f], x[f], a);
    h1[j] = a > 0.f ? a : 0.f;
  }
  for (int j = 0; j < H; ++j) {
    float a = P[o.b2 + j];
    for (int k = 0; k < H; ++k) a = fmaf(P[o.w2 + size_t(j) * H + k], h1[k], a);
    h2[j] = a > 0.f ? a : 0.f;
  }
  float y = P[o.b3];
  for (int j = 0; j < H; ++j) y = fmaf(P[o.w3 + j], h2[j], y);
  const float r = y - T[i];
  L[i] = r * r / float(n);
  const float dy = 2.f * r / float(n);
  float* g = G + size_t(i) * n_params(H);
  g[o.b3] = dy;
  for (int j = 0; j < H; ++j) {
    g[o.w3 + j] = dy * h2[j];
    d2[j] = h2[j] > 0.f ? dy * P[o.w3 + j] : 0.f;
    g[o.b2 + j] = d2[j];
  }
  for (int j = 0; j < H; ++j)
    for (int k = 0; k < H; ++k) g[o.w2 + size_t(j) * H + k] = d2[j] * h1[k];
  for (int k = 0; k < H; ++k) {
    float d1 = 0.f;
    if (h1[k] > 0.f)
      for (int j = 0; j < H; ++j) d1 = fmaf(P[o.w2 + size_t(j) * H + k], d2[j], d1);
    g[o.b1 + k] = d1;
    for (int f = 0; f < F; ++f) g[o.w1 + size_t(k) * F + f] = d1 * x[f];
  }
}

// Column sums in a fixed order: out[p] = sum_i G[i][p]; out_loss = sum_i L[i] (thread 0 of block 0).
__global__ void k_sum_rows(const float* __restrict__ G, int n, size_t np, float* __restrict__ out,
                           const float* __restrict__ L, float* __restrict__ out_loss) {
  const size_t p = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (p < np) {
    float s = 0.f;
    for (int i = 0; i < n; ++i) s += G[size_t(i) * np + p];
    out[p] = s;
  }
  if (p == 0 && out_loss) {
    float s = 0.f;
    for (int i = 0; i < n; ++i) s += L[i];
    *out_loss = s;
  }
}

__global__ void k_adam(float* __restrict__ P, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       size_t np, float lr, float b1, float b2, float eps, float c1, float c2) {
  const size_t p = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (p >= np) return;
  m[p] = b1 * m[p] + (1.f - b1) * g[p];
  v[p] = b2 * v[p] + (1.f - b2) * g[p] * g[p];
  P[p] -= lr * (m[p] / c1) / (sqrtf(v[p] / c2) + eps);
}

template <class T> struct DevBuf {
  T* p = nullptr;
  explicit DevBuf(size_t n) { QSVB_CK(cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1))); }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

// Splitmix-based deterministic init (He-uniform for weights, zero biases).
std::vector<float> init_params(int H, uint64_t seed) {
  std::vector<float> P(n_params(H), 0.f);
  const Offsets o = offsets(H);
  uint64_t s = seed;
  auto uni = [&]() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return float(double(z >> 11) * 0x1.0p-53) * 2.f - 1.f;
  };
  for (size_t i = 0; i < size_t(H) * F; ++i) P[o.w1 + i] = uni() * std::sqrt(6.f / F);
  for (size_t i = 0; i < size_t(H) * H; ++i) P[o.w2 + i] = uni() * std::sqrt(6.f / H);
  for (int i = 0; i < H; ++i) P[o.w3 + i] = uni() * std::sqrt(6.f / H);
  return P;
}

void check_hidden(uint32_t H) { QSVB_REQUIRE(H >= 4 && H <= uint32_t(kMaxHidden), "hidden width must be 4..128"); }

}  // namespace
}  // namespace qsvb

using namespace qsvb;

extern "C" {

int qsvb_costmodel_forward_backward(qsvb_ctx* c, const float* params, uint32_t hidden, const float* X,
                                    const float* t, size_t n, float* loss, float* grad) {
  try {
    QSVB_REQUIRE(c && params && X && t && loss && grad, "null pointer");
    check_hidden(hidden);
    QSVB_REQUIRE(n >= 1 && n <= (1u << 20), "sample count must be 1..2^20");
    QSVB_CK(cudaSetDevice(c->device));
    const int H = int(hidden);
    const size_t np = n_params(H);
    DevBuf<float> dP(np), dX(n * F), dT(n), dG(n * np), dL(n), dg(np), dl(1);
    QSVB_CK(cudaMemcpyAsync(dP.p, params, np * 4, cudaMemcpyHostToDevice, c->stream));
    QSVB_CK(cudaMemcpyAsync(dX.p, X, n * F * 4, cudaMemcpyHostToDevice, c->stream));
    QSVB_CK(cudaMemcpyAsync(dT.p, t, n * 4, cudaMemcpyHostToDevice, c->stream));
    k_mlp_fwd_bwd<<<unsigned((n + 127) / 128), 128, 0, c->stream>>>(dP.p, H, dX.p, dT.p, int(n), dG.p, dL.p);
    QSVB_CK(cudaGetLastError());
    k_sum_rows<<<unsigned((np + 255) / 256), 256, 0, c->stream>>>(dG.p, int(n), np, dg.p, dL.p, dl.p);
    QSVB_CK(cudaGetLastError());
    QSVB_CK(cudaMemcpyAsync(grad, dg.p, np * 4, cudaMemcpyDeviceToHost, c->stream));
    QSVB_CK(cudaMemcpyAsync(loss, dl.p, 4, cudaMemcpyDeviceToHost, c->stream));
    QSVB_CK(cudaStreamSynchronize(c->stream));
    return QSVB_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}

int qsvb_costmodel_train(qsvb_ctx* c, const float* features, const float* log2_seconds, size_t n, uint32_t hidden,
                         uint32_t epochs, float lr, uint64_t seed, float* final_loss) {
  try {
    QSVB_REQUIRE(c && features && log2_seconds, "null pointer");
    check_hidden(hidden);
    QSVB_REQUIRE(n >= 2 && n <= (1u << 20), "sample count must be 2..2^20");
    QSVB_REQUIRE(epochs >= 1 && epochs <= 100000, "epochs must be 1..100000");
    QSVB_CK(cudaSetDevice(c->device));
    const int H = int(hidden);
    const size_t np = n_params(H);
    // feature / target normalisation on the host
    MlpModel m;
    m.hidden = H;
    m.mean.assign(F, 0.f);
    m.scale.assign(F, 1.f);
    for (int f = 0; f < F; ++f) {
      double s = 0, s2 = 0;
      for (size_t i = 0; i < n; ++i) {
        s += features[i * F + f];
        s2 += double(features[i * F + f]) * features[i * F + f];
      }
      const double mu = s / n, var = std::max(0.0, s2 / n - mu * mu);
      m.mean[f] = float(mu);
      m.scale[f] = var > 1e-12 ? float(1.0 / std::sqrt(var)) : 1.f;
    }
    double ys = 0, ys2 = 0;
    for (size_t i = 0; i < n; ++i) {
      ys += log2_seconds[i];
      ys2 += double(log2_seconds[i]) * log2_seconds[i];
    }
    m.y_mean = float(ys / n);
    m.y_scale = float(std::sqrt(std::max(1e-12, ys2 / n - (ys / n) * (ys / n))));
    std::vector<float> X(n * F), T(n);
    for (size_t i = 0; i < n; ++i) {
      for (int f = 0; f < F; ++f) X[i * F + f] = (features[i * F + f] - m.mean[f]) * m.scale[f];
      T[i] = (log2_seconds[i] - m.y_mean) / m.y_scale;
    }
    std::vector<float> P = init_params(H, seed);
    DevBuf<float> dP(np), dX(n * F), dT(n), dG(n * np), dL(n), dg(np), dm(np), dv(np), dl(1);
    QSVB_CK(cudaMemcpyAsync(dP.p, P.data(), np * 4, cudaMemcpyHostToDevice, c->stream));
    QSVB_CK(cudaMemcpyAsync(dX.p, X.data(), n * F * 4, cudaMemcpyHostToDevice, c->stream));
    QSVB_CK(cudaMemcpyAsync(dT.p, T.data(), n * 4, cudaMemcpyHostToDevice, c->stream));
    QSVB_CK(cudaMemsetAsync(dm.p, 0, np * 4, c->stream));
    QSVB_CK(cudaMemsetAsync(dv.p, 0, np * 4, c->stream));
    const float b1 = 0.9f, b2 = 0.999f;
    double c1 = 1.0, c2 = 1.0;
    for (uint32_t e = 0; e < epochs; ++e) {
      k_mlp_fwd_bwd<<<unsigned((n + 127) / 128), 128, 0, c->stream>>>(dP.p, H, dX.p, dT.p, int(n), dG.p, dL.p);
      k_sum_rows<<<unsigned((np + 255) / 256), 256, 0, c->stream>>>(dG.p, int(n), np, dg.p, dL.p,
                                                                    e + 1 == epochs ? dl.p : nullptr);
      c1 *= b1;
      c2 *= b2;
      k_adam<<<unsigned((np + 255) / 256), 256, 0, c->stream>>>(dP.p, dg.p, dm.p, dv.p, np, lr, b1, b2, 1e-8f,
                                                                 float(1.0 - c1), float(1.0 - c2));
    }
    QSVB_CK(cudaGetLastError());
    QSVB_CK(cudaMemcpyAsync(P.data(), dP.p, np * 4, cudaMemcpyDeviceToHost, c->stream));
    float l = 0.f;
    QSVB_CK(cudaMemcpyAsync(&l, dl.p, 4, cudaMemcpyDeviceToHost, c->stream));
    QSVB_CK(cudaStreamSynchronize(c->stream));
    const Offsets o = offsets(H);
    m.w1.assign(P.begin() + o.w1, P.begin() + o.b1);
    m.b1.assign(P.begin() + o.b1, P.begin() + o.w2);
    m.w2.assign(P.begin() + o.w2, P.begin() + o.b2);
    m.b2.assign(P.begin() + o.b2, P.begin() + o.w3);
    m.w3.assign(P.begin() + o.w3, P.begin() + o.b3);
    m.b3.assign(P.begin() + o.b3, P.end());
    install_model(m);
    if (final_loss) *final_loss = l;
    return QSVB_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}

// Flat image of the installed model: [hidden, mean(F), scale(F), y_mean, y_scale, params...].
int qsvb_costmodel_get(float* out, size_t cap, size_t* needed) {
  try {
    const MlpModel& m = installed_model();
    QSVB_REQUIRE(needed != nullptr, "null size pointer");
    if (m.hidden == 0) {
      *needed = 0;
      return QSVB_OK;
    }
    const size_t np = n_params(m.hidden), total = 1 + 2 * F + 2 + np;
    *needed = total;
    if (!out) return QSVB_OK;
    QSVB_REQUIRE(cap >= total, "output buffer too small");
    size_t k = 0;
    out[k++] = float(m.hidden);
    for (int f = 0; f < F; ++f) out[k++] = m.mean[f];
    for (int f = 0; f < F; ++f) out[k++] = m.scale[f];
    out[k++] = m.y_mean;
    out[k++] = m.y_scale;
    for (const auto* v : {&m.w1, &m.b1, &m.w2, &m.b2, &m.w3, &m.b3})
      for (float x : *v) out[k++] = x;
    return QSVB_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}

int qsvb_costmodel_set(const float* img, size_t len) {
  try {
    if (!img || len == 0) {
      install_model(MlpModel{});
      return QSVB_OK;
    }
    const int H = int(img[0]);
    check_hidden(uint32_t(H));
    const size_t np = n_params(H), total = 1 + 2 * F + 2 + np;
    QSVB_REQUIRE(len == total, "model image has the wrong length for its hidden width");
    MlpModel m;
    m.hidden = H;
    size_t k = 1;
    m.mean.assign(img + k, img + k + F);
    k += F;
    m.scale.assign(img + k, img + k + F);
    k += F;
    m.y_mean = img[k++];
    m.y_scale = img[k++];
    const Offsets o = offsets(H);
    const float* P = img + k;
    m.w1.assign(P + o.w1, P + o.b1);
    m.b1.assign(P + o.b1, P + o.w2);
    m.w2.assign(P + o.w2, P + o.b2);
    m.b2.assign(P + o.b2, P + o.w3);
    m.w3.assign(P + o.w3, P + o.b3);
    m.b3.assign(P + o.b3, P + np);
    install_model(m);
    return QSVB_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}

// Host forward of the installed model (log2 seconds per feature row); fails when none is installed.
int qsvb_costmodel_predict(const float* features, size_t n, float* out_log2_seconds) {
  try {
    QSVB_REQUIRE(features && out_log2_seconds, "null pointer");
    const MlpModel& m = installed_model();
    QSVB_REQUIRE(m.hidden > 0, "no cost model installed");
    for (size_t i = 0; i < n; ++i) out_log2_seconds[i] = mlp_forward_host(m, features + i * F);
    return QSVB_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}

}  // extern "C"
