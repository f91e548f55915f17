// Dense k-qubit sweep (k = 4..6) on the 5th-generation tensor cores (tcgen05), complex64 state.
//
// The sweep is the contraction Y = U X, X the state viewed as 2^k gate rows x 2^(n-k) columns.
// It runs as a real GEMM on the embedding
//     [Yr; Yi] = W [Xr; Xi],   W = [[Ur, -Ui], [Ui, Ur]]   (2^(k+1) x 2^(k+1))
// with BF16 hi/lo split operands and an FP32 accumulator in tensor memory:
//     W X ~= Wlo Xhi + Whi Xlo + Whi Xhi      (x = hi + lo, hi = bf16(x), lo = bf16(x - hi))
// which keeps about 16 significant bits per product (relative error ~1e-5 per sweep).
//
// A tile is 2^k gate rows x 64 columns, the columns being the 6 lowest non-gate state bits, so
// every global access is a contiguous run of >= 64 amplitudes; tiles are disjoint and updated in
// place. One persistent CTA per SM runs a warp-specialized pipeline:
//   loader warps (8): keep R tiles of loads in flight in a register ring, split each tile into
//     bf16 hi/lo and store it into one of two B buffers (128-byte swizzle; MN-major when state
//     bits 0-1 are tile columns, K-major when they are the gate's two lowest qubits);
//   MMA warp (1, one elected lane): 3 * 2^(k+1)/16 tcgen05.mma per tile into one of two TMEM
//     accumulators (128 lanes x 64 fp32 columns); tcgen05.commit frees the B buffer and hands the
//     accumulator to the epilogue;
//   epilogue warps (4, one per TMEM lane quadrant): tcgen05.ld the accumulator, stage it in
//     address order (16-byte XOR swizzle), release the accumulator, then write the tile back with
//     coalesced 16-byte streaming stores.
// A (Whi, Wlo; M = 128 rows, K-major, 128-byte swizzle) is packed on the host in the exact
// shared-memory byte layout and copied in once per CTA. Every mbarrier wait is bounded: a wait
// that runs out sets the context error flag and that role stops; the host reports QSVB_E_TIMEOUT.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "qsvb_internal.h"

namespace qsvb {

namespace {

constexpr int kTcCols = 64;     // tile columns (N of the MMA)
constexpr int kTcColBits = 6;
constexpr int kLoadWarps = 8;
constexpr int kEpiWarps = 4;
constexpr int kLoadThreads = kLoadWarps * 32;
constexpr int kEpiThreads = kEpiWarps * 32;
constexpr int kTcThreads = kLoadThreads + 32 + kEpiThreads;  // loaders, MMA warp, epilogue
constexpr int kMmaWarp = kLoadWarps;                          // warp 8
constexpr int kEpiWarp0 = kLoadWarps + 1;                     // warps 9..12 (quadrants 1,2,3,0)
constexpr int kTmemCols = 128;                                // two 64-column accumulators
constexpr long long kWaitBudget = 1ll << 31;                  // clock64 cycles (~1 s)

struct TcParams {
  uint32_t hibits[6];      // tile bits above the 6 column bits (ascending)
  uint64_t hioff[64];      // address offset of the high tile bits
  uint16_t dsthi[64];      // (row << 6 | col) contribution of the high tile bits
  uint16_t dstlo[64];      // (row << 6 | col) contribution of the low 6 address bits
  uint16_t trow[64];       // address-order tile index of gate row s
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

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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

// Bounded wait for the phase with the given parity; false when the budget ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kWaitBudget) return false;
  return true;
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

__device__ __forceinline__ void named_sync(uint32_t id, uint32_t nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

__device__ __forceinline__ uint2 pack4(const __nv_bfloat16 (&x)[4]) {
  uint2 u;
  u.x = uint32_t(__bfloat16_as_ushort(x[0])) | (uint32_t(__bfloat16_as_ushort(x[1])) << 16);
  u.y = uint32_t(__bfloat16_as_ushort(x[2])) | (uint32_t(__bfloat16_as_ushort(x[3])) << 16);
  return u;
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

template <int KQ> struct TcShape {
  static constexpr int M2 = 1 << KQ;               // complex gate rows
  static constexpr int KR = 2 * M2;                // real rows (MMA K)
  static constexpr int KP = KR < 64 ? 64 : KR;     // padded K (one swizzle row = 64 elements)
  static constexpr uint32_t A_BYTES = 128u * KP * 2u;
  static constexpr uint32_t B_BYTES = 64u * KP * 2u;   // one of hi / lo
  static constexpr int TILE = M2 * kTcCols;        // complex amplitudes per tile
  static constexpr int VL = TILE / 4 / kLoadThreads;   // float4 per component per loader thread
  static constexpr int R = KQ == 6 ? 2 : (KQ == 5 ? 4 : 8);  // tiles in flight per loader
  static constexpr int VE = TILE / 4 / kEpiThreads;    // float4 per component per epilogue thread
  static constexpr size_t SMEM = 1024 + 2 * A_BYTES + 2 * (2 * B_BYTES) + size_t(TILE) * 8 + 128 + 64 * 8 + 4 * 64 * 2;
};

template <int KQ>
__global__ void __launch_bounds__(kTcThreads, 1) k_tc_dense(float* __restrict__ re, float* __restrict__ im,
                                                            uint64_t ntiles, const uint4* __restrict__ wpack,
                                                            TcParams p, int* err) {
  using S = TcShape<KQ>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* a_hi = smem;
  uint8_t* a_lo = a_hi + S::A_BYTES;
  uint8_t* bbuf = a_lo + S::A_BYTES;               // slot s: hi at bbuf + s*2*B, lo right after
  float* stage = reinterpret_cast<float*>(bbuf + 4 * S::B_BYTES);  // re [TILE] then im [TILE]
  uint64_t* bars = reinterpret_cast<uint64_t*>(stage + 2 * S::TILE);
  uint64_t* bfull = bars;        // [2] loaders -> MMA
  uint64_t* bfree = bars + 2;    // [2] MMA commit -> loaders
  uint64_t* dfull = bars + 4;    // [2] MMA commit -> epilogue
  uint64_t* dfree = bars + 6;    // [2] epilogue -> MMA
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 8);
  uint64_t* s_hioff = reinterpret_cast<uint64_t*>(bars + 16);
  uint16_t* s_dhi = reinterpret_cast<uint16_t*>(s_hioff + 64);
  uint16_t* s_dlo = s_dhi + 64;
  uint16_t* s_trow = s_dlo + 64;
  uint16_t* s_tcol = s_trow + 64;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  {
    uint4* dst = reinterpret_cast<uint4*>(a_hi);
    for (uint32_t i = tid; i < 2 * S::A_BYTES / 16; i += kTcThreads) dst[i] = wpack[i];
  }
  for (int i = tid; i < 64; i += kTcThreads) {
    s_hioff[i] = p.hioff[i];
    s_dhi[i] = p.dsthi[i];
    s_dlo[i] = p.dstlo[i];
    s_trow[i] = p.trow[i];
    s_tcol[i] = p.tcol[i];
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < 2; ++s) {
      mbar_init(&bfull[s], kLoadThreads);
      mbar_init(&bfree[s], 1);
      mbar_init(&dfull[s], 1);
      mbar_init(&dfree[s], kEpiThreads);
    }
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t b_mn = p.bmode == 0 ? 1u : 0u;

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
  const uint64_t my_tiles = uint64_t(blockIdx.x) < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  if (warp < kLoadWarps) {
    // ============================ loaders: global -> registers -> bf16 hi/lo B buffers
    float4 rr[S::R][S::VL], ri[S::R][S::VL];
    auto load = [&](uint64_t i, float4 (&xr)[S::VL], float4 (&xi)[S::VL]) {
      const uint64_t base = tile_base(blockIdx.x + i * gridDim.x);
#pragma unroll
      for (int j = 0; j < S::VL; ++j) {
        const int t = (tid + j * kLoadThreads) * 4, tlo = t & (kTcCols - 1), thi = t >> kTcColBits;
        const uint64_t a = base + s_hioff[thi] + uint64_t(tlo);
        xr[j] = __ldcs(reinterpret_cast<const float4*>(re + a));
        xi[j] = __ldcs(reinterpret_cast<const float4*>(im + a));
      }
    };
#pragma unroll
    for (int r = 0; r < S::R; ++r)
      if (uint64_t(r) < my_tiles) load(r, rr[r], ri[r]);
    bool ok = true;
    for (uint64_t i0 = 0; i0 < my_tiles && ok; i0 += S::R) {
#pragma unroll
      for (int r = 0; r < S::R; ++r) {
        const uint64_t i = i0 + r;
        if (i >= my_tiles || !ok) break;
        const uint32_t slot = uint32_t(i & 1), par = uint32_t((i >> 1) & 1);
        if (!mbar_wait(&bfree[slot], par ^ 1u)) {
          atomicExch(err, 1);
          ok = false;
          break;
        }
        uint8_t* b_hi = bbuf + slot * 2 * S::B_BYTES;
        uint8_t* b_lo = b_hi + S::B_BYTES;
#pragma unroll
        for (int j = 0; j < S::VL; ++j) {
          const int t = (tid + j * kLoadThreads) * 4, tlo = t & (kTcCols - 1), thi = t >> kTcColBits;
          const float vr[4] = {rr[r][j].x, rr[r][j].y, rr[r][j].z, rr[r][j].w};
          const float vi[4] = {ri[r][j].x, ri[r][j].y, ri[r][j].z, ri[r][j].w};
          if (p.bmode == 2) {
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const uint32_t d = uint32_t(s_dlo[tlo + e]) + s_dhi[thi];
              const uint32_t s = d >> 6, c = d & 63u;
              const uint32_t o_re = b_mn ? mnmaj_off(s, c) : kmaj_off(c, s, 64);
              const uint32_t o_im = b_mn ? mnmaj_off(s + S::M2, c) : kmaj_off(c, s + S::M2, 64);
              __nv_bfloat16 h, l;
              split_bf16(vr[e], h, l);
              *reinterpret_cast<__nv_bfloat16*>(b_hi + o_re) = h;
              *reinterpret_cast<__nv_bfloat16*>(b_lo + o_re) = l;
              split_bf16(vi[e], h, l);
              *reinterpret_cast<__nv_bfloat16*>(b_hi + o_im) = h;
              *reinterpret_cast<__nv_bfloat16*>(b_lo + o_im) = l;
            }
          } else {
            // four consecutive columns of row s (MN-major) or four consecutive rows of column c
            const uint32_t d = uint32_t(s_dlo[tlo]) + s_dhi[thi];
            const uint32_t s = d >> 6, c = d & 63u;
            const uint32_t o_re = b_mn ? mnmaj_off(s, c) : kmaj_off(c, s, 64);
            const uint32_t o_im = b_mn ? mnmaj_off(s + S::M2, c) : kmaj_off(c, s + S::M2, 64);
            __nv_bfloat16 hr[4], lr[4], hm[4], lm[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              split_bf16(vr[e], hr[e], lr[e]);
              split_bf16(vi[e], hm[e], lm[e]);
            }
            *reinterpret_cast<uint2*>(b_hi + o_re) = pack4(hr);
            *reinterpret_cast<uint2*>(b_lo + o_re) = pack4(lr);
            *reinterpret_cast<uint2*>(b_hi + o_im) = pack4(hm);
            *reinterpret_cast<uint2*>(b_lo + o_im) = pack4(lm);
          }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(&bfull[slot]);
        if (i + S::R < my_tiles) load(i + S::R, rr[r], ri[r]);
      }
    }
  } else if (warp == kMmaWarp) {
    // ============================ MMA issue: one lane
    if (lane == 0) {
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (b_mn << 16) | (uint32_t(kTcCols >> 3) << 17) |
                             (uint32_t(128 >> 4) << 24);
      const uint32_t a_hi_s = smem_u32(a_hi), a_lo_s = smem_u32(a_lo);
      for (uint64_t i = 0; i < my_tiles; ++i) {
        const uint32_t slot = uint32_t(i & 1), par = uint32_t((i >> 1) & 1);
        if (!mbar_wait(&bfull[slot], par) || !mbar_wait(&dfree[slot], par ^ 1u)) {
          atomicExch(err, 1);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t b_hi_s = smem_u32(bbuf + slot * 2 * S::B_BYTES), b_lo_s = b_hi_s + S::B_BYTES;
        const uint32_t d_tmem = tmem + slot * kTcCols;
#pragma unroll 1
        for (int s = 0; s < S::KR / 16; ++s) {
          const uint32_t ak = (s >> 2) * (128u * 128u) + (s & 3) * 32u;
          const uint32_t bk = b_mn ? uint32_t(s) * 2048u : (s >> 2) * (64u * 128u) + (s & 3) * 32u;
          const uint32_t b_lbo = b_mn ? uint32_t(S::KP) * 128u : 16u;
          const uint64_t dah = sw128_desc(a_hi_s + ak, 16u, 1024u), dal = sw128_desc(a_lo_s + ak, 16u, 1024u);
          const uint64_t dbh = sw128_desc(b_hi_s + bk, b_lbo, 1024u), dbl = sw128_desc(b_lo_s + bk, b_lbo, 1024u);
          mma_bf16(d_tmem, dal, dbh, idesc, s > 0 ? 1u : 0u);
          mma_bf16(d_tmem, dah, dbl, idesc, 1u);
          mma_bf16(d_tmem, dah, dbh, idesc, 1u);
        }
        mma_commit(&bfree[slot]);  // B buffer consumed
        mma_commit(&dfull[slot]);  // accumulator ready
      }
    }
    __syncwarp();
  } else {
    // ============================ epilogue: TMEM -> staging -> global
    const int ew = warp - kEpiWarp0;          // 0..3
    const int quad = warp & 3;                // TMEM lane quadrant this warp may access
    const int et = tid - kEpiWarp0 * 32;      // 0..127
    const uint32_t m = uint32_t(quad * 32 + lane);  // accumulator row = TMEM lane
    const bool has_row = int(m) < S::KR;
    const uint32_t s = m & uint32_t(S::M2 - 1), part = m >> KQ;
    (void)ew;
    for (uint64_t i = 0; i < my_tiles; ++i) {
      const uint32_t slot = uint32_t(i & 1), par = uint32_t((i >> 1) & 1);
      if (!mbar_wait(&dfull[slot], par)) {
        atomicExch(err, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      named_sync(1, kEpiThreads);  // the previous tile's write-back has finished reading staging
      if (quad * 32 < S::KR) {
        float* st = stage + part * S::TILE;
        const uint32_t tr = s_trow[s];
#pragma unroll 1
        for (int cb = 0; cb < kTcCols / 16; ++cb) {
          float v[16];
          tmem_ld16(tmem + (uint32_t(quad * 32) << 16) + slot * kTcCols + uint32_t(cb * 16), v);
          if (has_row) {
            if (p.bmode == 0) {
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                const uint32_t t = tr + s_tcol[cb * 16 + q * 4];
                *reinterpret_cast<float4*>(st + stage_idx(t)) =
                    make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
              }
            } else {
#pragma unroll
              for (int q = 0; q < 16; ++q) st[stage_idx(tr + s_tcol[cb * 16 + q])] = v[q];
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(&dfree[slot]);
      named_sync(1, kEpiThreads);  // staging complete
      const uint64_t base = tile_base(blockIdx.x + i * gridDim.x);
#pragma unroll
      for (int j = 0; j < S::VE; ++j) {
        const int t = (et + j * kEpiThreads) * 4, tlo = t & (kTcCols - 1), thi = t >> kTcColBits;
        const uint64_t a = base + s_hioff[thi] + uint64_t(tlo);
        const uint32_t si = stage_idx(uint32_t(t));
        __stcs(reinterpret_cast<float4*>(re + a), *reinterpret_cast<const float4*>(stage + si));
        __stcs(reinterpret_cast<float4*>(im + a), *reinterpret_cast<const float4*>(stage + S::TILE + si));
      }
    }
  }
  __syncwarp();  // roles may leave their loops at different iterations after a timeout
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
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
  return (s.kind == SK_DENSE || s.kind == SK_DENSE_TC) && s.m >= 4 && s.m <= 6 && n >= s.m + kTcColBits + 2 &&
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
  const size_t smem = TcShape<KQ>::SMEM;
  QSVB_CK(cudaFuncSetAttribute(k_tc_dense<KQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  QSVB_CK(cudaFuncSetAttribute(k_tc_dense<KQ>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               int(cudaSharedmemCarveoutMaxShared)));
  // one persistent CTA per SM (the tensor-memory allocation assumes it)
  const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(env.num_sms))));
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
