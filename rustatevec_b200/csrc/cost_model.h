// Sweep cost model used by the planner: an analytic roofline model, replaced by a small MLP once
// one has been trained on the autotuner's timing records (mlp.cu).
#pragma once

#include <vector>

#include "qsvb_internal.h"

namespace qsvb {

constexpr int kNumFeatures = 16;

// Feature vector of one sweep on an n-qubit state of precision dtype (inputs of the MLP).
void sweep_features(const Sweep& s, uint32_t n, int dtype, float* out);
// Roofline estimate (seconds).
double analytic_sweep_seconds(const Sweep& s, uint32_t n, int dtype);
// MLP estimate when a trained model is installed, else the analytic estimate.
double predict_sweep_seconds(const Sweep& s, uint32_t n, int dtype);
double predict_plan_seconds(const std::vector<Sweep>& sw, uint32_t n, int dtype);

// Kernel choice for dense sweeps (CUDA cores vs tensor cores), shared by the planner and the
// candidate evaluation of the learned planner.
void select_engines(std::vector<Sweep>& sw, uint32_t n, const qsvb_plan_opts& o, int dtype);

// Learned planner: cheapest candidate plan under the cost model.
std::vector<Gate> learned_fuse(const std::vector<Gate>& seg, uint32_t n, const qsvb_plan_opts& o, int dtype);

// Fusion strategies (planner.cpp).
// cost_only: groups whose sweep kind does not depend on their entries are left uncomposed (no
// matrix), for costing candidates; the chosen candidate is fused again with cost_only false.
std::vector<Gate> fuse_greedy_public(const std::vector<Gate>& in, uint32_t maxq, bool cost_only = false);
std::vector<Gate> fuse_window_public(const std::vector<Gate>& in, uint32_t maxq, bool cost_only = false);

// Installed MLP (weights are host copies; mlp.cu trains them on the device).
struct MlpModel {
  int hidden = 0;                   // 0 = no model installed
  std::vector<float> w1, b1, w2, b2, w3, b3;  // in->h, h->h, h->1
  std::vector<float> mean, scale;   // feature normalisation
  float y_mean = 0, y_scale = 1;    // target normalisation (log seconds)
};
const MlpModel& installed_model();
void install_model(const MlpModel& m);
float mlp_forward_host(const MlpModel& m, const float* feat);

}  // namespace qsvb
