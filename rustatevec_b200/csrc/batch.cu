// Batched execution of many small independent circuits (placeholder until the persistent runner
// lands): rejects the request so callers see a clear status.
#include "qsvb_internal.h"

void run_batch(qsvb_ctx*, const qsvb_circuit*, size_t, int, double*, double*, const uint64_t*, qsvb_plan_stats*) {
  throw qsvb::Error(QSVB_E_UNSUPPORTED, "batched execution is not available in this build");
}
