// Allocation-free <Z_mask> over caller-owned device buffers.
//
// Every other entry point works through a qsvb_ctx, whose creation reserves device scratch with
// cudaMalloc (reduction partials, matrix staging). Some callers cannot allow that: a host that runs
// a 33-qubit complex128 state (128 GiB) under a fixed device-memory budget, a framework that owns
// every device allocation through its own pool and forbids stray cudaMalloc calls, or a
// latency-sensitive loop that cannot afford the implicit device synchronization of cudaMalloc /
// cudaFree. For them, qsvb_expectation_z_noalloc runs the same FP64 reduction as
// qsvb_expectation_z with its scratch in a file-scope __device__ array instead:
//   - the array is kNoAllocScratchDoubles doubles (16.4 KB) and every GPU that loads the library
//     holds it until the process exits;
//   - it has room for the partial sums of at most kNoAllocMaxCtas CTAs; the entry point never
//     launches more and returns QSVB_E_INVALID for requests it cannot serve within that limit;
//   - all calls on a device share the array and it keeps the previous call's contents (each call
//     overwrites every slot it reads), so two calls whose kernels overlap on the GPU (different
//     streams, no ordering between them) race and may return wrong values;
//   - the first call on a device looks the array's device address up with cudaGetSymbolAddress
//     (the host-side symbol is only a stand-in for it); make that first call before any stream
//     capture begins. The address is kept per device together with the id of the CUDA context it
//     belongs to, so after a cudaDeviceReset the next call (in the new context) looks it up again;
//   - d_re and d_im must be device (or managed) memory of the current device, each 16-byte
//     aligned (the reduction reads them with 16-byte vector loads). Host pointers, memory of
//     another device and misaligned sub-buffer offsets are refused with QSVB_E_INVALID before any
//     kernel is launched.
// It calls no cudaMalloc, cudaFree or allocating library routine.

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include <mutex>
#include <string>

#include "qsvb_internal.h"

namespace qsvb {
namespace {

constexpr int kNoAllocMaxCtas = 1024;
constexpr int kNoAllocScratchDoubles = 2 * kNoAllocMaxCtas + 2;  // partial pairs + the result pair

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // id of the context the address belongs to

// Driver entry points through the runtime (the library does not link the driver library itself).
template <class F> F driver_fn(const char* name) {
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  QSVB_CK(cudaGetDriverEntryPoint(name, &fn, cudaEnableDefault, &q));
  QSVB_REQUIRE(q == cudaDriverEntryPointSuccess && fn != nullptr, std::string("driver entry point missing: ") + name);
  return reinterpret_cast<F>(fn);
}

// Id of the current CUDA context (unique for the life of the process; a context created after a
// cudaDeviceReset gets a new one).
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static const GetCurrent get_current = driver_fn<GetCurrent>("cuCtxGetCurrent");
  static const GetId get_id = driver_fn<GetId>("cuCtxGetId");
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  QSVB_REQUIRE(get_current(&ctx) == CUDA_SUCCESS && ctx != nullptr, "no current CUDA context");
  QSVB_REQUIRE(get_id(ctx, &id) == CUDA_SUCCESS, "cuCtxGetId failed");
  return id;
}

// Device address of the scratch array on the current device (set up once per device and context).
double* scratch_for(int dev) {
  QSVB_REQUIRE(dev >= 0 && dev < kMaxDevices, "device ordinal out of range");
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    QSVB_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_addr[dev] = static_cast<double*>(p);
    g_scratch_ctx[dev] = ctx;
  }
  return g_scratch_addr[dev];
}

// The caller's buffer must be device or managed memory of `dev`, 16-byte aligned.
void require_device_buffer(const void* p, int dev, const char* name) {
  QSVB_REQUIRE(reinterpret_cast<uintptr_t>(p) % 16 == 0, std::string(name) + " must be 16-byte aligned");
  cudaPointerAttributes a{};
  const cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();  // reset the runtime's last-error state that the failed query set
    throw Error(QSVB_E_INVALID, std::string(name) + " is not a CUDA pointer");
  }
  QSVB_REQUIRE(a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged,
               std::string(name) + " must be device or managed memory");
  QSVB_REQUIRE(a.device == dev, std::string(name) + " belongs to another device");
}

}  // namespace

}  // namespace qsvb

using namespace qsvb;

extern "C" int qsvb_expectation_z_noalloc(const void* d_re, const void* d_im, uint32_t n_qubits, int dtype,
                                          uint64_t mask, void* stream, double* out) {
  try {
    QSVB_REQUIRE(d_re && d_im && out, "null pointer");
    QSVB_REQUIRE(n_qubits >= 1 && n_qubits <= QSVB_MAX_QUBITS, "qubit count must be 1..34");
    QSVB_REQUIRE(dtype == QSVB_C64 || dtype == QSVB_C128, "dtype must be QSVB_C64 or QSVB_C128");
    int dev = 0, sms = 0;
    QSVB_CK(cudaGetDevice(&dev));
    QSVB_CK(cudaSetDevice(dev));  // makes the device's primary context current (no allocation)
    require_device_buffer(d_re, dev, "d_re");
    require_device_buffer(d_im, dev, "d_im");
    QSVB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    QSVB_REQUIRE(reduce_partials_needed(sms) <= size_t(2 * kNoAllocMaxCtas),
                 "device has more SMs than the allocation-free scratch (1024 partial sums) serves");
    double* scratch = scratch_for(dev);
    double* result = scratch + 2 * kNoAllocMaxCtas;
    const LaunchEnv env{static_cast<cudaStream_t>(stream), sms, nullptr};
    if (dtype == QSVB_C128)
      launch_reduce<double>(env, RED_EXPZ, static_cast<const double*>(d_re), static_cast<const double*>(d_im),
                            nullptr, nullptr, n_qubits, mask, scratch, result);
    else
      launch_reduce<float>(env, RED_EXPZ, static_cast<const float*>(d_re), static_cast<const float*>(d_im), nullptr,
                           nullptr, n_qubits, mask, scratch, result);
    double h[2];
    QSVB_CK(cudaMemcpyAsync(h, result, sizeof(h), cudaMemcpyDeviceToHost, env.stream));
    QSVB_CK(cudaStreamSynchronize(env.stream));
    *out = h[0];
    return QSVB_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return QSVB_E_INVALID;
  }
}
