// Dense k-qubit sweep (k = 4..6) on the 5th-generation tensor cores (tcgen05), complex64 state.
//
// The sweep is the contraction Y = U X, X the state viewed as 2^k gate rows x 2^(n-k) columns.
// It runs as a real GEMM on the embedding
//     [Yr; Yi] = W [Xr; Xi],   W = [[Ur, -Ui], [Ui, Ur]]   (2^(k+1) x 2^(k+1))
// with BF16 hi/lo split operands and an FP32 accumulator in tensor memory:
//     W X ~= Whi Xhi + Whi Xlo + Wlo Xhi      (x = hi + lo, hi = bf16(x), lo = bf16(x - hi))
// which keeps about 16 significant bits per product (relative error ~1e-5 per sweep).
//
// Per CTA (128 threads, persistent over tiles):
//   A (shared, loaded once): Whi and Wlo, M = 128 rows (rows >= 2^(k+1) are zero), K-major,
//     128-byte swizzle, packed on the host in exactly the shared-memory byte layout.
//   B (shared, per tile): the tile's 2^(k+1) real rows x 64 columns as bf16 hi and lo. The tile
//     columns are the 6 lowest non-gate state bits, so every global access is a contiguous run of
//     >= 64 amplitudes. B is MN-major when state bits 0-1 are column bits (a float4 load = 4
//     columns of one row) and K-major when they are the gate's two lowest qubits (4 rows of one
//     column); both use the 128-byte swizzle so the 8-byte stores of 4 bf16 are conflict-free.
//   D (tensor memory, 64 columns): 128 lanes (real rows) x 64 fp32 columns.
//   The result is staged in the (then free) B buffer in address order with a 16-byte XOR swizzle
//   and written back with coalesced 16-byte stores to the same addresses it was read from.
// One thread issues the 3 * 2^(k+1)/16 MMAs; tcgen05.commit arrives on an mbarrier that the CTA
// waits on with a bounded spin (a timeout sets an error flag and ends the CTA's loop).

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "qsvb_internal.h"

namespace qsvb {

namespace {

constexpr int kTcThreads = 128;
constexpr int kTcCols = 64;     // tile columns (N of the MMA)
constexpr int kTcColBits = 6;
constexpr int kTmemCols = 64;

struct TcParams {
  uint32_t hibits[6];      // tile bits above the 6 column bits (ascending)
  uint64_t hioff[64];      // address offset of the high tile bits
  uint16_t dsthi[64];      // (row << 6 | col) contribution of the high tile bits
  uint16_t dstlo[64];      // (row << 6 | col) contribution of the low 6 address bits
  uint16_t trow[64];       // address-order tile index of gate row s (0 for column bits)
  uint16_t tcol[64];       // address-order tile index of column c
  uint32_t bmode;          // 0: MN-major vector, 1: K-major vector, 2: scalar stores
};

// ----------------------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= uint64_t((addr >> 4) & 0x3FFFu);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;          // descriptor version for tcgen05
  d |= uint64_t(2) << 61;          // 128-byte swizzle
  return d;
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// Byte offset in a K-major, 128-byte-swizzled operand with `rows` rows (8-row atoms of 1024 B; a
// row of an atom holds 64 K-elements; 64-element K blocks follow each other every rows*128 B).
__device__ __forceinline__ uint32_t kmaj_off(uint32_t row, uint32_t kk, uint32_t rows) {
  return (kk >> 6) * (rows * 128u) + (row >> 3) * 1024u + (row & 7u) * 128u +
         ((((kk & 63u) >> 3) ^ (row & 7u)) << 4) + (kk & 7u) * 2u;
}
// Byte offset in an MN-major, 128-byte-swizzled operand of 64 columns (one atom wide).
__device__ __forceinline__ uint32_t mnmaj_off(uint32_t kk, uint32_t col) {
  return (kk >> 3) * 1024u + (kk & 7u) * 128u + ((((col >> 3) ^ (kk & 7u))) << 4) + (col & 7u) * 2u;
}
// Output staging (fp32, address order) with a 16-byte XOR swizzle against bank conflicts.
__device__ __forceinline__ uint32_t stage_idx(uint32_t t) { return t ^ (((t >> 7) & 7u) << 2); }

template <int KQ>
__global__ void __launch_bounds__(kTcThreads) k_tc_dense(float* __restrict__ re, float* __restrict__ im,
                                                         uint64_t ntiles, const uint4* __restrict__ wpack,
                                                         TcParams p, int* err) {
  constexpr int M2 = 1 << KQ;            // complex gate rows
  constexpr int KR = 2 * M2;             // real rows (MMA K)
  constexpr int KP = KR < 64 ? 64 : KR;  // padded K (one swizzle row = 64 elements)
  constexpr uint32_t A_BYTES = 128u * KP * 2u;
  constexpr uint32_t B_BYTES = 64u * KP * 2u;
  constexpr int TILE = M2 * kTcCols;     // complex amplitudes per tile
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* a_hi = smem;
  uint8_t* a_lo = a_hi + A_BYTES;
  uint8_t* b_hi = a_lo + A_BYTES;
  uint8_t* b_lo = b_hi + B_BYTES;
  float* stage = reinterpret_cast<float*>(b_hi);  // aliases B once the MMAs are done
  uint64_t* bar = reinterpret_cast<uint64_t*>(b_lo + B_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
  uint64_t* s_hioff = reinterpret_cast<uint64_t*>(tmem_slot + 2);
  uint16_t* s_dhi = reinterpret_cast<uint16_t*>(s_hioff + 64);
  uint16_t* s_dlo = s_dhi + 64;
  uint16_t* s_trow = s_dlo + 64;
  uint16_t* s_tcol = s_trow + 64;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  {
    const uint4* src = wpack;
    uint4* dst = reinterpret_cast<uint4*>(a_hi);
    for (uint32_t i = tid; i < 2 * A_BYTES / 16; i += kTcThreads) dst[i] = src[i];
  }
  for (int i = tid; i < 64; i += kTcThreads) {
    s_hioff[i] = p.hioff[i];
    s_dhi[i] = p.dsthi[i];
    s_dlo[i] = p.dstlo[i];
    s_trow[i] = p.trow[i];
    s_tcol[i] = p.tcol[i];
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // instruction descriptor: D f32, A/B bf16, A K-major, B MN- or K-major, N = 64, M = 128
  const uint32_t b_mn = p.bmode == 0 ? 1u : 0u;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (b_mn << 16) | (uint32_t(kTcCols >> 3) << 17) |
                         (uint32_t(128 >> 4) << 24);
  const uint32_t a_hi_s = smem_u32(a_hi), a_lo_s = smem_u32(a_lo), b_hi_s = smem_u32(b_hi), b_lo_s = smem_u32(b_lo);

  uint32_t phase = 0;
  bool failed = false;
  // Each thread owns V float4 of each component per tile. The next tile's loads are issued right
  // after the current tile's MMAs, so they are in flight during the MMA wait, the epilogue and the
  // write-back (32 KB per CTA for k = 6).
  constexpr int V = TILE / 4 / kTcThreads;
  auto tile_base = [&](uint64_t tile) {
    uint64_t base = tile << kTcColBits;
#pragma unroll
    for (int j = 0; j < KQ; ++j) {
      const uint32_t b = p.hibits[j];
      const uint64_t lo = base & ((1ull << b) - 1ull);
      base = ((base - lo) << 1) | lo;
    }
    return base;
  };
  float4 pr[V], pim[V];
  auto load_tile = [&](uint64_t base) {
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int t = (tid + j * kTcThreads) * 4, tlo = t & (kTcCols - 1), thi = t >> kTcColBits;
      const uint64_t a = base + s_hioff[thi] + uint64_t(tlo);
      pr[j] = __ldcs(reinterpret_cast<const float4*>(re + a));
      pim[j] = __ldcs(reinterpret_cast<const float4*>(im + a));
    }
  };
  if (uint64_t(blockIdx.x) < ntiles) load_tile(tile_base(blockIdx.x));
  for (uint64_t tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
    const uint64_t base = tile_base(tile);
    // ---- split the prefetched tile into B (bf16 hi/lo)
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int t = (tid + j * kTcThreads) * 4, tlo = t & (kTcCols - 1), thi = t >> kTcColBits;
      const float4 xr = pr[j], xi = pim[j];
      const float vr[4] = {xr.x, xr.y, xr.z, xr.w}, vi[4] = {xi.x, xi.y, xi.z, xi.w};
      if (p.bmode == 2) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const uint32_t d = uint32_t(s_dlo[tlo + e]) + s_dhi[thi];
          const uint32_t s = d >> 6, c = d & 63u;
          __nv_bfloat16 h, l;
          const uint32_t o_re = b_mn ? mnmaj_off(s, c) : kmaj_off(c, s, 64);
          const uint32_t o_im = b_mn ? mnmaj_off(s + M2, c) : kmaj_off(c, s + M2, 64);
          split_bf16(vr[e], h, l);
          *reinterpret_cast<__nv_bfloat16*>(b_hi + o_re) = h;
          *reinterpret_cast<__nv_bfloat16*>(b_lo + o_re) = l;
          split_bf16(vi[e], h, l);
          *reinterpret_cast<__nv_bfloat16*>(b_hi + o_im) = h;
          *reinterpret_cast<__nv_bfloat16*>(b_lo + o_im) = l;
        }
      } else {
        const uint32_t d = uint32_t(s_dlo[tlo]) + s_dhi[thi];
        const uint32_t s = d >> 6, c = d & 63u;
        // four consecutive columns of row s (MN-major) or four consecutive rows of column c (K-major)
        const uint32_t o_re = b_mn ? mnmaj_off(s, c) : kmaj_off(c, s, 64);
        const uint32_t o_im = b_mn ? mnmaj_off(s + M2, c) : kmaj_off(c, s + M2, 64);
        __nv_bfloat16 hr[4], lr[4], hm[4], lm[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          split_bf16(vr[e], hr[e], lr[e]);
          split_bf16(vi[e], hm[e], lm[e]);
        }
        auto pack = [](const __nv_bfloat16 (&x)[4]) {
          uint2 u;
          u.x = uint32_t(__bfloat16_as_ushort(x[0])) | (uint32_t(__bfloat16_as_ushort(x[1])) << 16);
          u.y = uint32_t(__bfloat16_as_ushort(x[2])) | (uint32_t(__bfloat16_as_ushort(x[3])) << 16);
          return u;
        };
        *reinterpret_cast<uint2*>(b_hi + o_re) = pack(hr);
        *reinterpret_cast<uint2*>(b_lo + o_re) = pack(lr);
        *reinterpret_cast<uint2*>(b_hi + o_im) = pack(hm);
        *reinterpret_cast<uint2*>(b_lo + o_im) = pack(lm);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // ---- MMAs: D = Wlo Xhi + Whi Xlo + Whi Xhi over K = 2^(k+1) in steps of 16
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
      for (int s = 0; s < KR / 16; ++s) {
        const uint32_t ak = (s >> 2) * (128u * 128u) + (s & 3) * 32u;
        const uint32_t bk = b_mn ? uint32_t(s) * 2048u : (s >> 2) * (64u * 128u) + (s & 3) * 32u;
        const uint32_t b_lbo = b_mn ? uint32_t(KP) * 128u : 16u;
        const uint64_t dah = sw128_desc(a_hi_s + ak, 16u, 1024u), dal = sw128_desc(a_lo_s + ak, 16u, 1024u);
        const uint64_t dbh = sw128_desc(b_hi_s + bk, b_lbo, 1024u), dbl = sw128_desc(b_lo_s + bk, b_lbo, 1024u);
        mma_bf16(tmem, dal, dbh, idesc, s > 0 ? 1u : 0u);
        mma_bf16(tmem, dah, dbl, idesc, 1u);
        mma_bf16(tmem, dah, dbh, idesc, 1u);
      }
      mma_commit(bar);
    }
    // ---- prefetch the next tile while the tensor cores work
    if (tile + gridDim.x < ntiles) load_tile(tile_base(tile + gridDim.x));
    // ---- bounded wait for the MMAs
    {
      const long long t0 = clock64();
      bool ok = false;
      while (!ok) {
        ok = mbar_try_wait(bar, phase);
        if (!ok && clock64() - t0 > (1ll << 32)) break;
      }
      failed = __syncthreads_or(ok ? 0 : 1) != 0;  // one decision for the whole CTA
      if (failed && tid == 0) atomicExch(err, 1);
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (failed) break;
    // ---- epilogue: TMEM -> staging (address order, swizzled), warps own 32 real rows each
    if (warp * 32 < KR) {
      const uint32_t m = uint32_t(warp * 32 + lane);
      const uint32_t s = m & uint32_t(M2 - 1), part = m >> KQ;
      float* st = stage + part * TILE;
      const uint32_t tr = s_trow[s];
#pragma unroll 1
      for (int cb = 0; cb < kTcCols / 16; ++cb) {
        float v[16];
        tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(cb * 16), v);
        if (p.bmode == 0) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const uint32_t t = tr + s_tcol[cb * 16 + q * 4];
            *reinterpret_cast<float4*>(st + stage_idx(t)) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
          }
        } else {
#pragma unroll
          for (int q = 0; q < 16; ++q) st[stage_idx(tr + s_tcol[cb * 16 + q])] = v[q];
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // ---- coalesced write-back to the addresses the tile came from
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int t = (tid + j * kTcThreads) * 4, tlo = t & (kTcCols - 1), thi = t >> kTcColBits;
      const uint64_t a = base + s_hioff[thi] + uint64_t(tlo);
      const uint32_t si = stage_idx(uint32_t(t));
      __stcs(reinterpret_cast<float4*>(re + a), *reinterpret_cast<const float4*>(stage + si));
      __stcs(reinterpret_cast<float4*>(im + a), *reinterpret_cast<const float4*>(stage + TILE + si));
    }
    __syncthreads();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

template <int KQ> constexpr size_t tc_smem_bytes() {
  constexpr int KR = 2 << KQ, KP = KR < 64 ? 64 : KR;
  return 1024 /*alignment slack*/ + 2 * 128 * KP * 2 + 2 * 64 * KP * 2 + 16 + 64 * 8 + 4 * 64 * 2;
}

// ---------------------------------------------------------------- host-side packing of W
uint16_t bf16_bits_rn(float x) {  // round-to-nearest-even, finite inputs
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return uint16_t(u >> 16);
}
float bf16_to_float(uint16_t h) {
  const uint32_t u = uint32_t(h) << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
uint32_t kmaj_off_host(uint32_t row, uint32_t kk, uint32_t rows) {
  return (kk >> 6) * (rows * 128u) + (row >> 3) * 1024u + (row & 7u) * 128u +
         ((((kk & 63u) >> 3) ^ (row & 7u)) << 4) + (kk & 7u) * 2u;
}

}  // namespace

bool tc_dense_supported(const Sweep& s, uint32_t n) {
  return (s.kind == SK_DENSE || s.kind == SK_DENSE_TC) && s.m >= 4 && s.m <= 6 && n >= s.m + kTcColBits &&
         n >= 12;
}

size_t tc_matrix_bytes(const Sweep& s) {
  const size_t KR = size_t(2) << s.m, KP = std::max<size_t>(64, KR);
  return 2 * 128 * KP * 2;
}

// W = [[Ur, -Ui], [Ui, Ur]] split into bf16 hi/lo, K-major, 128-byte swizzle, 128 rows.
void tc_pack_matrix(const Sweep& s, void* dst) {
  const uint32_t M2 = 1u << s.m, KR = 2 * M2, KP = std::max<uint32_t>(64, KR);
  const size_t a_bytes = size_t(128) * KP * 2;
  uint8_t* hi = static_cast<uint8_t*>(dst);
  uint8_t* lo = hi + a_bytes;
  std::memset(dst, 0, 2 * a_bytes);
  for (uint32_t r = 0; r < KR; ++r)
    for (uint32_t k = 0; k < KR; ++k) {
      const cd u = s.mat[size_t(r % M2) * M2 + (k % M2)];
      double w;
      if (r < M2) w = k < M2 ? u.real() : -u.imag();
      else w = k < M2 ? u.imag() : u.real();
      const uint16_t h = bf16_bits_rn(float(w));
      const uint16_t l = bf16_bits_rn(float(w - double(bf16_to_float(h))));
      const uint32_t o = kmaj_off_host(r, k, 128);
      std::memcpy(hi + o, &h, 2);
      std::memcpy(lo + o, &l, 2);
    }
}

template <int KQ>
static void launch_tc_k(const LaunchEnv& env, float* re, float* im, uint32_t n, const Sweep& s, const void* dev_mat) {
  constexpr int M2 = 1 << KQ;
  TcParams p{};
  int gate_rank[64], col_rank[64];
  for (int b = 0; b < 64; ++b) gate_rank[b] = col_rank[b] = -1;
  for (int j = 0; j < KQ; ++j) gate_rank[s.q[j]] = j;
  std::vector<uint32_t> tbits;
  int ncol = 0;
  for (uint32_t b = 0; b < n; ++b) {
    if (gate_rank[b] >= 0) tbits.push_back(b);
    else if (ncol < kTcColBits) {
      col_rank[b] = ncol++;
      tbits.push_back(b);
    }
  }
  for (int j = 0; j < kTcColBits; ++j) QSVB_REQUIRE(tbits[j] == uint32_t(j), "tc tile: low bits not contiguous");
  auto contrib = [&](uint32_t b) -> uint32_t {
    return gate_rank[b] >= 0 ? (uint32_t(1) << gate_rank[b]) << kTcColBits : (uint32_t(1) << col_rank[b]);
  };
  for (int j = 0; j < KQ; ++j) p.hibits[j] = tbits[kTcColBits + j];
  for (int h = 0; h < M2; ++h) {
    uint64_t off = 0;
    uint32_t d = 0;
    for (int j = 0; j < KQ; ++j)
      if ((h >> j) & 1) {
        off |= 1ull << p.hibits[j];
        d += contrib(p.hibits[j]);
      }
    p.hioff[h] = off;
    p.dsthi[h] = uint16_t(d);
  }
  for (int l = 0; l < kTcCols; ++l) {
    uint32_t d = 0;
    for (int b = 0; b < kTcColBits; ++b)
      if ((l >> b) & 1) d += contrib(uint32_t(b));
    p.dstlo[l] = uint16_t(d);
  }
  // address-order tile index of each gate row / column: tile position = rank among tile bits
  for (int sidx = 0; sidx < M2; ++sidx) {
    uint32_t t = 0;
    for (int j = 0; j < KQ; ++j)
      if ((sidx >> j) & 1) t |= 1u << uint32_t(std::find(tbits.begin(), tbits.end(), s.q[j]) - tbits.begin());
    p.trow[sidx] = uint16_t(t);
  }
  for (int c = 0; c < kTcCols; ++c) {
    uint32_t t = 0;
    for (uint32_t b = 0; b < n; ++b)
      if (col_rank[b] >= 0 && ((c >> col_rank[b]) & 1))
        t |= 1u << uint32_t(std::find(tbits.begin(), tbits.end(), b) - tbits.begin());
    p.tcol[c] = uint16_t(t);
  }
  const bool low_cols = gate_rank[0] < 0 && gate_rank[1] < 0;
  const bool low_rows = gate_rank[0] == 0 && gate_rank[1] == 1;
  p.bmode = low_cols ? 0u : (low_rows ? 1u : 2u);

  const uint64_t ntiles = 1ull << (n - KQ - kTcColBits);
  const size_t smem = tc_smem_bytes<KQ>();
  QSVB_CK(cudaFuncSetAttribute(k_tc_dense<KQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  int occ = 1;
  QSVB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tc_dense<KQ>, kTcThreads, smem));
  occ = std::max(1, std::min(occ, 512 / kTmemCols));  // tensor-memory columns per SM bound the CTAs
  const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(env.num_sms) * occ)));
  k_tc_dense<KQ><<<grid, kTcThreads, smem, env.stream>>>(re, im, ntiles, static_cast<const uint4*>(dev_mat), p,
                                                         env.err_flag);
  QSVB_CK(cudaGetLastError());
}

void launch_tc_dense(const LaunchEnv& env, float* re, float* im, uint32_t n, const Sweep& s, const void* dev_mat) {
  QSVB_REQUIRE(tc_dense_supported(s, n), "tensor-core sweep: unsupported shape");
  QSVB_REQUIRE(env.err_flag != nullptr, "tensor-core sweep needs the context error flag");
  switch (s.m) {
    case 4: launch_tc_k<4>(env, re, im, n, s, dev_mat); break;
    case 5: launch_tc_k<5>(env, re, im, n, s, dev_mat); break;
    case 6: launch_tc_k<6>(env, re, im, n, s, dev_mat); break;
    default: throw Error(QSVB_E_INVALID, "tensor-core sweep arity must be 4..6");
  }
}

}  // namespace qsvb
