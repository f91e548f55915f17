// Tensor-core dense sweep (placeholder until the tcgen05 kernel lands): reports unsupported so
// the planner keeps every dense sweep on CUDA cores.
#include "qsvb_internal.h"

namespace qsvb {

bool tc_dense_supported(const Sweep&, uint32_t) { return false; }
size_t tc_matrix_bytes(const Sweep&) { return 0; }
void tc_pack_matrix(const Sweep&, void*) {}
void launch_tc_dense(const LaunchEnv&, float*, float*, uint32_t, const Sweep&, const void*) {
  throw Error(QSVB_E_UNSUPPORTED, "tensor-core sweeps are not available in this build");
}

}  // namespace qsvb
