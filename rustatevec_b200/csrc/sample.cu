// Measurement sampling on the device: shots drawn from the state's outcome distribution without
// downloading it, by the inverse-CDF rule of qsv's cdf_sample (crates/qsv-core/src/sample.rs:163-172).
//
// Shot k takes the k-th `unit()` value of SplitMix64(seed) (crates/qsv-core/src/circuits.rs:22-46),
// u_k in [0, 1), scales it by the total probability, x_k = u_k * total, and returns the first
// outcome i whose cumulative probability CDF(i) >= x_k (cdf_sample's `partition_point(|&c| c < u)`,
// a lower bound; the last outcome if rounding leaves none). The probabilities are |amp|^2 computed
// as the trait's `probabilities` does, in the state's precision (re*re + im*im, no fused
// multiply-add), and accumulated in FP64; the device sums them in another order than the
// reference's chunked scan, so a draw can differ only where x_k lies within rounding of a CDF value.
// Steps: the FP64 total of each 8192-amplitude block; an exclusive scan of those; the scaled
// uniforms sorted with their shot numbers; then one pass over the blocks: block b takes the sorted
// values x with CDFstart(b) < x <= CDFstart(b + 1) (block 0 also x = 0), builds its inclusive
// prefix in shared memory and places each shot by binary search, writing the outcome at the shot's
// original position.

#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>

#include "qsvb_internal.h"

namespace qsvb {
namespace {

constexpr int kBlockBits = 13;
constexpr int kSampleThreads = 512;

template <class T> struct DevBuf {
  T* p = nullptr;
  explicit DevBuf(size_t n) { QSVB_CK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T))); }
  ~DevBuf() { cudaFree(p); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

// |amp|^2 rounded as StateVector::probabilities computes it in the state's precision
// (crates/qsv-core/src/state/mod.rs:130-134: re*re + im*im with separate roundings), widened to FP64.
__device__ __forceinline__ double prob_of(float x, float y) {
  return double(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)));
}
__device__ __forceinline__ double prob_of(double x, double y) { return __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)); }

__device__ __forceinline__ uint64_t mix64s(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// FP64 sum of |amp|^2 over each block of 2^bb amplitudes (one block per CTA iteration).
template <class R>
__global__ void __launch_bounds__(kSampleThreads) k_block_sums(const R* __restrict__ re, const R* __restrict__ im,
                                                               uint32_t bb, uint64_t nblocks,
                                                               double* __restrict__ bsum) {
  __shared__ double s_red[kSampleThreads / 32];
  const uint32_t B = 1u << bb;
  for (uint64_t b = blockIdx.x; b < nblocks; b += gridDim.x) {
    double acc = 0.0;
    for (uint32_t i = threadIdx.x; i < B; i += kSampleThreads) {
      const uint64_t a = (b << bb) + i;
      acc += prob_of(re[a], im[a]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < kSampleThreads / 32; ++w) s += s_red[w];
      bsum[b] = s;
    }
    __syncthreads();
  }
}

// Scaled uniforms as sortable keys (non-negative doubles order like their bit patterns).
__global__ void k_uniforms(uint64_t shots, uint64_t seed, const double* __restrict__ bcdf,
                           const double* __restrict__ bsum, uint64_t nblocks, uint64_t* __restrict__ keys,
                           uint64_t* __restrict__ vals) {
  const double total = bcdf[nblocks - 1] + bsum[nblocks - 1];
  const uint64_t G = 0x9E3779B97F4A7C15ull;
  for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < shots; k += uint64_t(gridDim.x) * blockDim.x) {
    const double u = double(mix64s(seed + (k + 1) * G) >> 11) * 0x1.0p-53;
    keys[k] = __double_as_longlong(u * total);
    vals[k] = k;
  }
}

// First index of the sorted keys whose value is > x.
__device__ __forceinline__ uint64_t upper_bound_keys(const uint64_t* __restrict__ keys, uint64_t n, double x) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (__longlong_as_double(keys[mid]) <= x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Each block that holds shots (the sorted scaled uniforms in (bcdf[b], bcdf[b+1]]; block 0 from
// 0 inclusive) scans its probabilities (FP64, inclusive) and places its shots.
template <class R>
__global__ void __launch_bounds__(kSampleThreads) k_assign(const R* __restrict__ re, const R* __restrict__ im,
                                                           uint32_t bb, uint64_t nblocks,
                                                           const double* __restrict__ bcdf,
                                                           const double* __restrict__ bsum,
                                                           const uint64_t* __restrict__ keys,
                                                           const uint64_t* __restrict__ vals, uint64_t shots,
                                                           uint64_t* __restrict__ out) {
  extern __shared__ double s_pre[];  // 2^bb inclusive prefix sums
  __shared__ double s_warp[kSampleThreads / 32];
  __shared__ uint64_t s_range[2];
  const uint32_t B = 1u << bb;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (uint64_t b = blockIdx.x; b < nblocks; b += gridDim.x) {
    if (tid == 0) {
      s_range[0] = b == 0 ? 0 : upper_bound_keys(keys, shots, bcdf[b]);
      s_range[1] = b + 1 == nblocks ? shots : upper_bound_keys(keys, shots, bcdf[b + 1]);
    }
    __syncthreads();
    const uint64_t j0 = s_range[0], j1 = s_range[1];
    if (j1 > j0) {
      // this thread's run of consecutive amplitudes (B / threads of them, or one when B is small)
      const uint32_t per = B >= uint32_t(kSampleThreads) ? B / kSampleThreads : 1u;
      const uint32_t first = uint32_t(tid) * per;
      double run = 0.0;
      if (first < B)
        for (uint32_t e = 0; e < per; ++e) {
          const uint64_t a = (b << bb) + first + e;
          run += prob_of(re[a], im[a]);
          s_pre[first + e] = run;
        }
      // exclusive scan of the run totals across the block
      double incl = run;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      if (lane == 31) s_warp[warp] = incl;
      __syncthreads();
      if (warp == 0) {
        double w = lane < kSampleThreads / 32 ? s_warp[lane] : 0.0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const double v = __shfl_up_sync(0xffffffffu, w, o);
          if (lane >= o) w += v;
        }
        if (lane < kSampleThreads / 32) s_warp[lane] = w;
      }
      __syncthreads();
      const double off = (incl - run) + (warp > 0 ? s_warp[warp - 1] : 0.0);
      if (first < B)
        for (uint32_t e = 0; e < per; ++e) s_pre[first + e] += off;
      __syncthreads();
      const double base = bcdf[b];
      for (uint64_t j = j0 + tid; j < j1; j += kSampleThreads) {
        const double x = __longlong_as_double(keys[j]);
        // the first index whose cumulative probability base + prefix is >= x (the block's last
        // one if none: rounding can leave x just above the block's own total)
        uint32_t lo = 0, hi = B - 1;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (__dadd_rn(base, s_pre[mid]) >= x) hi = mid;
          else lo = mid + 1;
        }
        // in that clamped case, step back over trailing zero probabilities
        if (__dadd_rn(base, s_pre[lo]) < x)
          while (lo > 0 && s_pre[lo] == s_pre[lo - 1]) --lo;
        out[vals[j]] = (b << bb) + lo;
      }
    }
    __syncthreads();
  }
}

template <class R>
void sample_impl(qsvb_ctx* c, const qsvb_state* st, uint64_t shots, uint64_t seed, uint64_t* out_host) {
  const uint32_t n = st->n_qubits;
  const uint32_t bb = std::min<uint32_t>(n, kBlockBits);
  const uint64_t nblocks = uint64_t(1) << (n - bb);
  const R* re = static_cast<const R*>(st->re);
  const R* im = static_cast<const R*>(st->im);
  cudaStream_t s = c->stream;
  DevBuf<double> bsum(nblocks), bcdf(nblocks);
  DevBuf<uint64_t> keys(shots), vals(shots), keys2(shots), vals2(shots), out(shots);
  const int grid = int(std::min<uint64_t>(nblocks, uint64_t(c->num_sms) * 4));
  k_block_sums<R><<<grid, kSampleThreads, 0, s>>>(re, im, bb, nblocks, bsum.p);
  QSVB_CK(cudaGetLastError());
  size_t tb_scan = 0, tb_sort = 0;
  QSVB_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, bsum.p, bcdf.p, nblocks, s));
  QSVB_CK(cub::DeviceRadixSort::SortPairs(nullptr, tb_sort, keys.p, keys2.p, vals.p, vals2.p, shots, 0, 64, s));
  DevBuf<char> temp(std::max(tb_scan, tb_sort));
  QSVB_CK(cub::DeviceScan::ExclusiveSum(temp.p, tb_scan, bsum.p, bcdf.p, nblocks, s));
  k_uniforms<<<c->num_sms * 8, 256, 0, s>>>(shots, seed, bcdf.p, bsum.p, nblocks, keys.p, vals.p);
  QSVB_CK(cudaGetLastError());
  QSVB_CK(cub::DeviceRadixSort::SortPairs(temp.p, tb_sort, keys.p, keys2.p, vals.p, vals2.p, shots, 0, 64, s));
  const size_t smem = sizeof(double) << bb;
  QSVB_CK(cudaFuncSetAttribute(k_assign<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  k_assign<R><<<grid, kSampleThreads, smem, s>>>(re, im, bb, nblocks, bcdf.p, bsum.p, keys2.p, vals2.p, shots,
                                                 out.p);
  QSVB_CK(cudaGetLastError());
  d2h_staged(c, out_host, out.p, shots * sizeof(uint64_t));
}

}  // namespace

void sample_shots(qsvb_ctx* c, const qsvb_state* st, uint64_t shots, uint64_t seed, uint64_t* out) {
  QSVB_REQUIRE(out != nullptr, "null output");
  QSVB_REQUIRE(shots >= 1 && shots <= (uint64_t(1) << 30), "shots must be 1..2^30");
  if (st->dtype == QSVB_C128) sample_impl<double>(c, st, shots, seed, out);
  else sample_impl<float>(c, st, shots, seed, out);
}

}  // namespace qsvb
