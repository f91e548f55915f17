// Dense k-qubit sweep (k = 4..6) on the 5th-generation tensor cores (tcgen05), complex64 state.
//
// The sweep is the contraction Y = U X, X the state viewed as 2^k gate rows x 2^(n-k) columns.
// It runs as a real GEMM on the embedding
//     [Yr; Yi] = W [Xr; Xi],   W = [[Ur, -Ui], [Ui, Ur]]   (KR x KR, KR = 2^(k+1))
// with BF16 hi/lo split operands and an FP32 accumulator in tensor memory:
//     W X ~= Wlo Xhi + Whi Xlo + Whi Xhi      (x = hi + lo, hi = bf16(x), lo = bf16(x - hi))
// which keeps about 16 significant bits per product (relative error ~1e-5 per sweep).
//
// Every k uses the same MMA shape, M = 128, K = 128, N = 64: the A operand is W repeated
// nblk = 128 / KR times on the diagonal, and the B operand stacks nblk blocks of 64 state
// columns along K. A tile is therefore always 4096 amplitudes (2^k gate rows x 64 * nblk
// columns, the columns being the 12 - k lowest non-gate state bits, so every global access is a
// contiguous run of >= 64 amplitudes) and all 128 accumulator lanes carry results.
//
// One persistent CTA per SM runs a warp-specialized pipeline over its tiles:
//   producer warp: one tiled TMA (a tensor map whose dimensions are the runs of tile bits) or
//     bulk copies (cp.async.bulk, one per contiguous run; no multicast anywhere) of the tile's
//     re/im into one of four fp32 input slots, completing on that slot's mbarrier;
//   converter warps (8): split the staged tile into bf16 hi/lo and store it into one of two B
//     buffers (128-byte swizzle; the layout is a template parameter: MN-major when state bits 0-1
//     are tile columns, K-major when they are the gate's two lowest qubits, K-major assembled by
//     lane-pair shuffles when bit 0 is a column and bit 1 the gate's lowest qubit, K-major row
//     pairs otherwise), then release the input slot to the producer;
//   MMA warp (1 lane): 24 tcgen05.mma per tile into one of two TMEM accumulators (128 lanes x
//     64 fp32 columns); tcgen05.commit frees the B buffer and hands the accumulator on;
//   epilogue warps (4, one per TMEM lane quadrant): tcgen05.ld the accumulator, release it, write
//     the result into the output staging buffer (address order, 16-byte XOR swizzle) and write
//     the tile back with coalesced 16-byte streaming stores.
// A (Whi, Wlo; K-major, 128-byte swizzle) is packed on the host in the exact shared-memory byte
// layout and copied in once per CTA. Every mbarrier wait is bounded: a wait that runs out sets the
// context error flag and that role stops (the epilogue threads vote before their named barriers,
// so they stop together); the host reports QSVB_E_TIMEOUT.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "qsvb_internal.h"
#include "tc_common.cuh"

namespace qsvb {

namespace {
using namespace tc;

constexpr int kMmaN = 64;                 // MMA N: columns per block
constexpr int kMmaK = 128;                // MMA K (real rows, all blocks)
constexpr int kTileAmps = 4096;           // complex amplitudes per tile
constexpr int kTileBits = 12;
constexpr int kCvtWarps = 8;
constexpr int kEpiWarps = 4;
constexpr int kCvtThreads = kCvtWarps * 32;
constexpr int kEpiThreads = kEpiWarps * 32;
constexpr int kProdWarp = kCvtWarps;                          // warp 8
constexpr int kMmaWarp = kCvtWarps + 1;                       // warp 9
constexpr int kEpiWarp0 = kCvtWarps + 2;                      // warps 10..13 (lane quadrants 2,3,0,1)
constexpr int kTcThreads = (kCvtWarps + 2 + kEpiWarps) * 32;
constexpr int kBSlots = 2;
constexpr int kIoSlots = 4;                 // input tiles in flight (released once converted)
constexpr int kIoBufs = kIoSlots + 1;       // + the epilogue's output staging
constexpr int kTmemCols = 256;                                // two 64-column accumulators + Whi + Wlo
constexpr uint32_t kTmemAHi = 128, kTmemALo = 192;           // A operand columns (64 each)
constexpr int kVC = kTileAmps / 4 / kCvtThreads;              // float4 per component per converter
constexpr int kVE = kTileAmps / 4 / kEpiThreads;              // float4 per component per epilogue thread
constexpr uint32_t kABytes = 128u * kMmaK * 2u;               // one of Whi / Wlo (global image)
constexpr uint32_t kBBytes = uint32_t(kMmaN) * kMmaK * 2u;    // one of Xhi / Xlo
constexpr uint32_t kIoBytes = kTileAmps * 8u;                 // re [4096] + im [4096] fp32
constexpr size_t kTcSmem = 1024 + kBSlots * 2 * size_t(kBBytes) + kIoBufs * size_t(kIoBytes) +
                           144 + 64 * 8 + 3 * 64 * 2 + 256 * 2 + 64 * 2;
static_assert(kTcSmem <= 232448, "tensor-core sweep: shared memory above the 227 KB per-block limit");

struct TcParams {
  uint32_t hibits[6];      // tile bits above the 6 lowest state bits (ascending)
  uint32_t ncb;            // column bits (12 - k)
  uint32_t runbits;        // log2 of the contiguous run length of a tile (>= 6)
  uint64_t hioff[64];      // address offset of the high tile bits
  uint16_t dsthi[64];      // (row << ncb | col) contribution of the high tile bits
  uint16_t dstlo[64];      // (row << ncb | col) contribution of the low 6 state bits
  uint16_t trow[64];       // address-order tile index of gate row s
  uint16_t tcol[256];      // address-order tile index of column c
  uint32_t bmode;          // 0: MN-major vector, 1: K-major vector, 2: K-major row pairs,
                           // 3: K-major vector assembled from a lane pair
  uint32_t b2_bit0;        // bmode 2: state bit 0 is the gate bit (else state bit 1 is)
  uint32_t pair_shift;     // bmode 3: the gate's second row bit is state bit pair_shift + 2
  // converter work order: float4 u (u = thread + j * converter threads) covers tile amplitudes
  // 4 * (tplo[u & 31] | tphi[u >> 5]): a bit permutation chosen on the host so that a warp's
  // K-major B stores fall in distinct banks (the identity for MN-major tiles)
  uint16_t tplo[32], tphi[32];
  uint32_t tcl[16];        // stage_idx(tcol[q]) for q < 16 (uniform; read straight from the parameter bank)
  uint32_t tclb[16];       // the same as byte offsets (K-major epilogue stores)
  uint32_t tm_rank;        // > 0: the producer uses one tensor-map TMA per component per tile
  uint32_t tm_start[5];    // first state bit of each tensor dimension
  uint32_t tm_len[5];      // bits of that dimension (a run of tile bits plus the run of non-tile bits above it)
  uint32_t tm_outer;       // tile bits folded into the last dimension (one copy per value)
  uint32_t tm_obit[3];     // their bit positions in that dimension's coordinate
};

// BM: the B-operand layout mode (TcParams::bmode), fixed at compile time so that each
// instantiation's converter loop holds only its own path.
template <int KQ, int BM>
__global__ void __launch_bounds__(kTcThreads, 1) k_tc_dense(float* __restrict__ re, float* __restrict__ im,
                                                            uint64_t ntiles, const uint4* __restrict__ wpack,
                                                            TcParams p, int* err, long long* prof,
                                                            const __grid_constant__ CUtensorMap tm_re,
                                                            const __grid_constant__ CUtensorMap tm_im) {
  constexpr int M2 = 1 << KQ;      // complex gate rows
  constexpr int KR = 2 * M2;       // real rows of one block
  constexpr int NCB = kTileBits - KQ;
  constexpr uint32_t CMASK = (1u << NCB) - 1u;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* bbuf = smem;                            // slot s: hi at bbuf + s*2*B, lo right after
  float* io = reinterpret_cast<float*>(bbuf + kBSlots * 2 * kBBytes);  // slot s: re [4096], im [4096]
  float* ostage = io + kIoSlots * 2 * kTileAmps;  // the epilogue's result, re [4096] then im [4096]
  uint64_t* bars = reinterpret_cast<uint64_t*>(io + kIoBufs * 2 * kTileAmps);
  uint64_t* iofull = bars;       // [4] TMA complete_tx -> converters
  uint64_t* ioempty = bars + 4;  // [4] converters -> producer
  uint64_t* bfull = bars + 8;    // [2] converters -> MMA
  uint64_t* bfree = bars + 10;   // [2] MMA commit -> converters
  uint64_t* dfull = bars + 12;   // [2] MMA commit -> epilogue
  uint64_t* dfree = bars + 14;   // [2] epilogue -> MMA
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 16);
  uint64_t* s_hioff = reinterpret_cast<uint64_t*>(bars + 18);
  uint16_t* s_dhi = reinterpret_cast<uint16_t*>(s_hioff + 64);
  uint16_t* s_dlo = s_dhi + 64;
  uint16_t* s_trow = s_dlo + 64;
  uint16_t* s_tcol = s_trow + 64;  // 256 entries
  uint16_t* s_tperm = s_tcol + 256;  // tplo [32] then tphi [32]

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long t_start = clock64();
  long long w0 = 0, w1 = 0, w2 = 0, w3 = 0, w4 = 0;  // per-role stall counters (stall profiling only)
  for (int i = tid; i < 64; i += kTcThreads) {
    s_hioff[i] = p.hioff[i];
    s_dhi[i] = p.dsthi[i];
    s_dlo[i] = p.dstlo[i];
    s_trow[i] = p.trow[i];
  }
  for (int i = tid; i < 256; i += kTcThreads) s_tcol[i] = p.tcol[i];
  for (int i = tid; i < 32; i += kTcThreads) {
    s_tperm[i] = p.tplo[i];
    s_tperm[32 + i] = p.tphi[i];
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < kIoSlots; ++s) {
      mbar_init(&iofull[s], 1);
      mbar_init(&ioempty[s], kCvtThreads);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&bfull[s], kCvtThreads);
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
  constexpr uint32_t b_mn = BM == 0 ? 1u : 0u;
  if (warp >= kEpiWarp0) {
    // A (Whi, Wlo) into tensor memory: the thread owning TMEM lane m writes row m of each, 64
    // 32-bit columns of packed bf16 pairs (element 2j in the low half).
    const uint32_t quad = uint32_t(warp & 3), m = quad * 32 + uint32_t(lane);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint32_t r[64];
      const uint4* src = wpack + (size_t(h) * 128 + m) * 16;
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const uint4 u = src[q];
        r[4 * q] = u.x;
        r[4 * q + 1] = u.y;
        r[4 * q + 2] = u.z;
        r[4 * q + 3] = u.w;
      }
      tmem_st64(tmem + ((quad * 32) << 16) + (h == 0 ? kTmemAHi : kTmemALo), r);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  auto tile_base = [&](uint64_t tile) {
    uint64_t base = tile << 6;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const uint32_t b = p.hibits[j];
      const uint64_t lo = base & ((1ull << b) - 1ull);
      base = ((base - lo) << 1) | lo;
    }
    return base;
  };
  // this CTA's tiles (an epilogue whose checked tables fail sets it to 0)
  uint64_t my_tiles = uint64_t(blockIdx.x) < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  if (warp == kProdWarp) {
    // ============================ producer: TMA bulk copies of the tile's contiguous runs
    const uint32_t rb = p.runbits, nruns = uint32_t(kTileAmps) >> rb, run_bytes = 4u << rb;
    for (uint64_t i = 0; i < my_tiles; ++i) {
      const uint32_t slot = uint32_t(i % kIoSlots), par = uint32_t((i / kIoSlots) & 1);
      bool ok = true;
      if (lane == 0) {
        ok = mbar_wait_t(&ioempty[slot], par ^ 1u, w0);
        if (ok) mbar_arrive_expect_tx(&iofull[slot], kIoBytes);
        else atomicOr(err, kErrTimeout);
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
      const uint64_t base = tile_base(blockIdx.x + i * gridDim.x);
      float* dre = io + slot * 2 * kTileAmps;
      float* dim_ = dre + kTileAmps;
      if (p.tm_rank > 0) {
        if (lane == 0)
          tma_tile_g2s(dre, dim_, &tm_re, &tm_im, base, p.tm_rank, p.tm_start, p.tm_len, p.tm_outer, p.tm_obit,
                       &iofull[slot]);
        continue;
      }
      for (uint32_t j = lane; j < nruns; j += 32) {
        const uint32_t t0 = j << rb;
        const uint64_t a = base + s_hioff[t0 >> 6];
        if (!QSVB_BC(a + (1ull << rb) <= (ntiles << 12), err)) continue;
        bulk_g2s(dre + t0, re + a, run_bytes, &iofull[slot]);
        bulk_g2s(dim_ + t0, im + a, run_bytes, &iofull[slot]);
      }
    }
  } else if (warp < kCvtWarps) {
    // ============================ converters: staged fp32 -> bf16 hi/lo B buffers
    for (uint64_t i = 0; i < my_tiles; ++i) {
      const uint32_t slot = uint32_t(i % kIoSlots), par = uint32_t((i / kIoSlots) & 1);
      const uint32_t bs = uint32_t(i & 1), bpar = uint32_t((i >> 1) & 1);
      const bool ready = mbar_wait_t(&iofull[slot], par, w0) && mbar_wait_t(&bfree[bs], bpar ^ 1u, w1);
      if (!__all_sync(0xffffffffu, ready)) {  // warp-uniform exit: the lane-pair mode shuffles
        atomicOr(err, kErrTimeout);
        break;
      }
      const float* sre = io + slot * 2 * kTileAmps;
      const float* sim = sre + kTileAmps;
      uint8_t* b_hi = bbuf + bs * 2 * kBBytes;
      uint8_t* b_lo = b_hi + kBBytes;
      // all shared-memory loads first (the B stores below could alias them for the compiler)
      float4 xra[kVC], xia[kVC];
      uint32_t dda[kVC];
      int tt[kVC];
#pragma unroll
      for (int j = 0; j < kVC; ++j) {
        const uint32_t u = uint32_t(tid + j * kCvtThreads);
        const int t0 = int(uint32_t(s_tperm[u & 31u]) | uint32_t(s_tperm[32 + (u >> 5)])) * 4;
        const int t = QSVB_BC(t0 + 4 <= kTileAmps, err) ? t0 : 0;
        tt[j] = t;
        xra[j] = *reinterpret_cast<const float4*>(sre + t);
        xia[j] = *reinterpret_cast<const float4*>(sim + t);
        dda[j] = uint32_t(s_dlo[t & 63]) + s_dhi[t >> 6];
      }
#pragma unroll
      for (int j = 0; j < kVC; ++j) {
        const int t = tt[j], tlo = t & 63, thi = t >> 6;
        const float4 xr = xra[j], xi = xia[j];
        const float vr[4] = {xr.x, xr.y, xr.z, xr.w};
        const float vi[4] = {xi.x, xi.y, xi.z, xi.w};
        if constexpr (BM == 3) {
          // state bit 0 is a column, bit 1 the gate's row bit 0 and state bit 2 + pair_shift its
          // row bit 1, which is lane bit pair_shift (the work order keeps float4 index bits 0..2
          // as lane bits 0..2). The lane pair differing in it holds rows 0-3 of two columns: each
          // lane gives its partner the two values of the partner's column and keeps four
          // consecutive rows of its own, stored like bmode 1.
          const uint32_t sh = p.pair_shift;
          const bool odd = ((uint32_t(lane) >> sh) & 1u) != 0;
          const int pm = 1 << sh;
          const float rr0 = __shfl_xor_sync(0xffffffffu, odd ? xr.x : xr.y, pm);
          const float rr1 = __shfl_xor_sync(0xffffffffu, odd ? xr.z : xr.w, pm);
          const float ri0 = __shfl_xor_sync(0xffffffffu, odd ? xi.x : xi.y, pm);
          const float ri1 = __shfl_xor_sync(0xffffffffu, odd ? xi.z : xi.w, pm);
          const float wr[4] = {odd ? rr0 : xr.x, odd ? rr1 : xr.z, odd ? xr.y : rr0, odd ? xr.w : rr1};
          const float wi[4] = {odd ? ri0 : xi.x, odd ? ri1 : xi.z, odd ? xi.y : ri0, odd ? xi.w : ri1};
          const int tg = (t & ~(4 << sh)) | (odd ? 1 : 0);  // the group's row-0 element of this column
          const uint32_t d = uint32_t(s_dlo[tg & 63]) + s_dhi[tg >> 6];
          const uint32_t s = d >> NCB, c = d & CMASK;
          const uint32_t kb = (c >> 6) * KR, cl = c & 63u;
          const uint32_t o_re = kmaj_off(cl, kb + s, 64);
          const uint32_t o_im = kmaj_off(cl, kb + M2 + s, 64);
          __nv_bfloat16 hr[4], lr[4], hm[4], lm[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            split_bf16(wr[e], hr[e], lr[e]);
            split_bf16(wi[e], hm[e], lm[e]);
          }
          if (QSVB_BC(o_re + 8 <= kBBytes && o_im + 8 <= kBBytes, err)) {
            *reinterpret_cast<uint2*>(b_hi + o_re) = pack4(hr);
            *reinterpret_cast<uint2*>(b_lo + o_re) = pack4(lr);
            *reinterpret_cast<uint2*>(b_hi + o_im) = pack4(hm);
            *reinterpret_cast<uint2*>(b_lo + o_im) = pack4(lm);
          }
        } else if constexpr (BM == 2) {
          // exactly one of state bits 0, 1 is a gate bit (the gate's lowest, so row parity): the
          // four amplitudes are two pairs of adjacent rows (K) in two columns, stored as bf16 pairs
          const int step = p.b2_bit0 ? 1 : 2;  // element offset of a pair's second row
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int e = p.b2_bit0 ? 2 * q : q;
            const uint32_t d = uint32_t(s_dlo[tlo + e]) + s_dhi[thi];
            const uint32_t s = d >> NCB, c = d & CMASK;
            const uint32_t kb = (c >> 6) * KR, cl = c & 63u;
            const uint32_t o_re = kmaj_off(cl, kb + s, 64);
            const uint32_t o_im = kmaj_off(cl, kb + M2 + s, 64);
            if (!QSVB_BC(o_re + 4 <= kBBytes && o_im + 4 <= kBBytes, err)) continue;
            __nv_bfloat16 h0, l0, h1, l1;
            split_bf16(vr[e], h0, l0);
            split_bf16(vr[e + step], h1, l1);
            *reinterpret_cast<uint32_t*>(b_hi + o_re) =
                uint32_t(__bfloat16_as_ushort(h0)) | (uint32_t(__bfloat16_as_ushort(h1)) << 16);
            *reinterpret_cast<uint32_t*>(b_lo + o_re) =
                uint32_t(__bfloat16_as_ushort(l0)) | (uint32_t(__bfloat16_as_ushort(l1)) << 16);
            split_bf16(vi[e], h0, l0);
            split_bf16(vi[e + step], h1, l1);
            *reinterpret_cast<uint32_t*>(b_hi + o_im) =
                uint32_t(__bfloat16_as_ushort(h0)) | (uint32_t(__bfloat16_as_ushort(h1)) << 16);
            *reinterpret_cast<uint32_t*>(b_lo + o_im) =
                uint32_t(__bfloat16_as_ushort(l0)) | (uint32_t(__bfloat16_as_ushort(l1)) << 16);
          }
        } else {
          // four consecutive columns of row s (MN-major) or four consecutive rows of column c
          const uint32_t d = dda[j];
          const uint32_t s = d >> NCB, c = d & CMASK;
          const uint32_t kb = (c >> 6) * KR, cl = c & 63u;
          const uint32_t o_re = b_mn ? mnmaj_off(kb + s, cl) : kmaj_off(cl, kb + s, 64);
          const uint32_t o_im = b_mn ? mnmaj_off(kb + M2 + s, cl) : kmaj_off(cl, kb + M2 + s, 64);
          __nv_bfloat16 hr[4], lr[4], hm[4], lm[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            split_bf16(vr[e], hr[e], lr[e]);
            split_bf16(vi[e], hm[e], lm[e]);
          }
          if (QSVB_BC(o_re + 8 <= kBBytes && o_im + 8 <= kBBytes, err)) {
            *reinterpret_cast<uint2*>(b_hi + o_re) = pack4(hr);
            *reinterpret_cast<uint2*>(b_lo + o_re) = pack4(lr);
            *reinterpret_cast<uint2*>(b_hi + o_im) = pack4(hm);
            *reinterpret_cast<uint2*>(b_lo + o_im) = pack4(lm);
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&bfull[bs]);
      mbar_arrive(&ioempty[slot]);  // this thread's reads of the input slot are done (fenced above)
    }
  } else if (warp == kMmaWarp) {
    // ============================ MMA issue: the whole warp walks the tiles (uniform operands), one
    // elected lane issues
    {
      const uint32_t leader = elect_one();
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (b_mn << 16) | (uint32_t(kMmaN >> 3) << 17) |
                             (uint32_t(128 >> 4) << 24);
      const uint32_t b_lbo = b_mn ? uint32_t(kMmaK) * 128u : 16u;
      for (uint64_t i = 0; i < my_tiles; ++i) {
        const uint32_t bs = uint32_t(i & 1), par = uint32_t((i >> 1) & 1);
        const bool ok = mbar_wait_t(&bfull[bs], par, w0) && mbar_wait_t(&dfree[bs], par ^ 1u, w1);
        if (!__all_sync(0xffffffffu, ok)) {
          if (leader) atomicOr(err, kErrTimeout);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d_tmem = tmem + bs * kMmaN;
        // descriptors of K step 0; step s adds its byte offset (>> 4) to the address field
        const uint64_t dbh0 = sw128_desc(smem_u32(bbuf + bs * 2 * kBBytes), b_lbo, 1024u);
        const uint64_t dbl0 = dbh0 + (kBBytes >> 4);
#pragma unroll
        for (int s = 0; s < kMmaK / 16; ++s) {
          const uint64_t o = (b_mn ? uint64_t(s) * 2048u : uint64_t((s >> 2) * (64 * 128) + (s & 3) * 32)) >> 4;
          const uint32_t tah = tmem + kTmemAHi + uint32_t(s) * 8u, tal = tmem + kTmemALo + uint32_t(s) * 8u;
          mma_bf16_ts_by(leader, d_tmem, tal, dbh0 + o, idesc, s > 0 ? 1u : 0u);
          mma_bf16_ts_by(leader, d_tmem, tah, dbl0 + o, idesc, 1u);
          mma_bf16_ts_by(leader, d_tmem, tah, dbh0 + o, idesc, 1u);
        }
        mma_commit_by(leader, &bfree[bs]);  // B buffer consumed
        mma_commit_by(leader, &dfull[bs]);  // accumulator ready
      }
    }
    __syncwarp();
  } else {
    // ============================ epilogue: TMEM -> the tile's staging slot -> global
    const int quad = warp & 3;                      // TMEM lane quadrant this warp may access
    const int et = tid - kEpiWarp0 * 32;            // 0..127
    const uint32_t m = uint32_t(quad * 32 + lane);  // accumulator row = TMEM lane
    const uint32_t blk = m / KR, r = m % KR;
    const uint32_t s = r & uint32_t(M2 - 1), part = r >> KQ;
    // address-order index of (row s, column blk*64 + cb*16 + q) = tr + tch[cb] + tcl[q]: the row
    // and column maps are bit deposits onto disjoint bits, so the sum is an XOR and its staging
    // index is stage_idx(tr ^ tch[cb]) ^ stage_idx(tcol[q]) (the latter precomputed in p.tcl)
    const uint32_t tr = s_trow[s];
    uint32_t sch[4];
#pragma unroll
    // MN-major layouts index floats; K-major ones use byte offsets (one fewer instruction per
    // scalar store, measured 3-6 % faster there; the MN-major instantiations spill with them)
    for (int cb = 0; cb < 4; ++cb)
      sch[cb] = (BM == 0 ? 1u : 4u) * stage_idx(tr ^ uint32_t(s_tcol[blk * 64 + cb * 16]));
    {
      // (checked builds) every staging offset of this thread, once; a failing epilogue stops and
      // the sweep ends through the other roles' bounded waits
      bool tables_ok = true;
      for (int cb = 0; cb < 4; ++cb)
        for (int q = 0; q < 16; ++q)
          tables_ok = tables_ok && QSVB_BC(BM == 0 ? (q % 4 == 0 ? (sch[cb] ^ p.tcl[q]) + 4 <= uint32_t(kTileAmps) : true)
                                                   : (sch[cb] ^ p.tclb[q]) + 4 <= uint32_t(kTileAmps) * 4u,
                                           err);
      if (!named_all(3, kEpiThreads, tables_ok)) my_tiles = 0;
    }
    for (uint64_t i = 0; i < my_tiles; ++i) {
      const uint32_t ds = uint32_t(i & 1), dpar = uint32_t((i >> 1) & 1);
      const bool ready = mbar_wait_t(&dfull[ds], dpar, w0);
      // one decision for all epilogue threads (they meet at named barriers below); reaching this
      // barrier also means every thread's reads of the previous tile's staging are done
      if (!named_all(2, kEpiThreads, ready)) {
        atomicOr(err, kErrTimeout);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const long long ta = clock64();
      uint32_t v[64];  // column c of this lane's accumulator row
      tmem_ld64_wait(tmem + (uint32_t(quad * 32) << 16) + ds * kMmaN, v);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(&dfree[ds]);  // accumulator may be overwritten now
      const long long tb = clock64();
      w2 += tb - ta;
      float* st = ostage + part * kTileAmps;
      if constexpr (BM == 0) {
#pragma unroll
        for (int cb = 0; cb < 4; ++cb)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            *reinterpret_cast<float4*>(st + (sch[cb] ^ p.tcl[q * 4])) =
                make_float4(__uint_as_float(v[cb * 16 + 4 * q]), __uint_as_float(v[cb * 16 + 4 * q + 1]),
                            __uint_as_float(v[cb * 16 + 4 * q + 2]), __uint_as_float(v[cb * 16 + 4 * q + 3]));
          }
      } else {
#pragma unroll
        for (int cb = 0; cb < 4; ++cb)
#pragma unroll
          for (int q = 0; q < 16; ++q)
            *reinterpret_cast<float*>(reinterpret_cast<char*>(st) + (sch[cb] ^ p.tclb[q])) = __uint_as_float(v[cb * 16 + q]);
      }
      const long long tc0 = clock64();
      w3 += tc0 - tb;
      named_sync(1, kEpiThreads);  // the whole result is staged
      const long long ts = clock64();
      w4 += ts - tc0;
      const float* sre = ostage;
      const uint64_t base = tile_base(blockIdx.x + i * gridDim.x);
#pragma unroll
      for (int j = 0; j < kVE; ++j) {
        const int t = (et + j * kEpiThreads) * 4, tlo = t & 63, thi = t >> 6;
        const uint64_t a = base + s_hioff[thi] + uint64_t(tlo);
        const uint32_t si = stage_idx(uint32_t(t));
        if (!QSVB_BC(a + 4 <= (ntiles << 12), err)) continue;
        __stcs(reinterpret_cast<float4*>(re + a), *reinterpret_cast<const float4*>(sre + si));
        __stcs(reinterpret_cast<float4*>(im + a), *reinterpret_cast<const float4*>(sre + kTileAmps + si));
      }
      w1 += clock64() - ts;
    }
  }
  if (prof != nullptr) {  // [producer, converter x2, MMA x2, epilogue x5, total] per CTA
    long long* pc = prof + 12 * blockIdx.x;
    if (warp == kProdWarp && lane == 0) pc[0] = w0;
    if (tid == 0) {
      pc[1] = w0;
      pc[2] = w1;
    }
    if (warp == kMmaWarp && lane == 0) {
      pc[3] = w0;
      pc[4] = w1;
    }
    if (tid == kEpiWarp0 * 32) {
      pc[5] = w0;
      pc[6] = w1;
      pc[7] = clock64() - t_start;
      pc[8] = w2;
      pc[9] = w3;
      pc[10] = w4;
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

}  // namespace

bool tc_dense_supported(const Sweep& s, uint32_t n) {
  return (s.kind == SK_DENSE || s.kind == SK_DENSE_TC) && s.m >= 4 && s.m <= 6 && n >= uint32_t(kTileBits);
}

size_t tc_matrix_bytes(const Sweep&) { return 2 * size_t(kABytes); }

// A = blockdiag(W, ..., W) (128 / KR copies), W = [[Ur, -Ui], [Ui, Ur]], split into bf16 hi/lo.
// Image for tensor memory: hi then lo, each 128 rows x 64 32-bit words, word j of row m holding
// elements (2j, 2j+1) of that row (2j in the low half).
void tc_pack_matrix(const Sweep& s, void* dst) {
  const uint32_t M2 = 1u << s.m, KR = 2 * M2, nblk = 128 / KR;
  uint16_t* hi = static_cast<uint16_t*>(dst);
  uint16_t* lo = hi + 128 * 128;
  std::memset(dst, 0, 2 * size_t(kABytes));
  for (uint32_t b = 0; b < nblk; ++b)
    for (uint32_t r = 0; r < KR; ++r)
      for (uint32_t k = 0; k < KR; ++k) {
        const cd u = s.mat[size_t(r % M2) * M2 + (k % M2)];
        double w;
        if (r < M2) w = k < M2 ? u.real() : -u.imag();
        else w = k < M2 ? u.imag() : u.real();
        const uint16_t h = bf16_bits_rn(float(w));
        const uint16_t l = bf16_bits_rn(float(w - double(bf16_to_float(h))));
        const size_t o = size_t(b * KR + r) * 128 + (b * KR + k);
        hi[o] = h;
        lo[o] = l;
      }
}

void tile_layout(uint32_t n, const uint32_t (&tbits)[12], float* re, float* im, TileLayout& out) {
  out = TileLayout{};
  std::memset(out.maps, 0, sizeof(out.maps));
  bool in_tile[64] = {false};
  for (int i = 0; i < 12; ++i) {
    QSVB_REQUIRE(tbits[i] < n && (i == 0 || tbits[i] > tbits[i - 1]), "tile bits must be ascending state bits");
    in_tile[tbits[i]] = true;
  }
  for (int j = 0; j < 6; ++j) QSVB_REQUIRE(tbits[j] == uint32_t(j), "tc tile: low bits not contiguous");
  for (int j = 0; j < 6; ++j) out.hibits[j] = tbits[6 + j];
  for (int h = 0; h < 64; ++h) {
    uint64_t off = 0;
    for (int j = 0; j < 6; ++j)
      if ((h >> j) & 1) off |= 1ull << out.hibits[j];
    out.hioff[h] = off;
  }
  uint32_t rb = 0;
  while (rb < uint32_t(kTileBitsAll) && tbits[rb] == rb) ++rb;
  out.runbits = rb;
  // Short runs: view the state as a tensor with one dimension per run of tile bits, each extended
  // by the run of non-tile bits above it. The box covers the tile part of every dimension and the
  // tile's coordinates are the base's bits (its tile bits are zero), so one tiled TMA per
  // component fetches the whole tile in address order.
  if (rb > 8) return;
  struct Dim {
    uint32_t start, tile_len, len;
  };
  std::vector<Dim> dims;
  for (uint32_t b = 0; b < n;) {
    uint32_t e = b;
    while (e < n && in_tile[e]) ++e;   // tile run [b, e)
    uint32_t f = e;
    while (f < n && !in_tile[f]) ++f;  // non-tile run above it [e, f)
    dims.push_back({b, e - b, f - b});
    b = f;
  }
  // A tensor map has at most five dimensions: fold every dimension above the fifth into it. Their
  // tile bits become bits of the fifth coordinate, fetched by one copy per value (at most two bits:
  // seven dimensions mean six single-bit runs of high tile bits).
  uint32_t obits[3] = {0, 0, 0}, nob = 0;
  bool ok = true;
  if (dims.size() > 5) {
    for (size_t d = 5; d < dims.size(); ++d)
      for (uint32_t t = 0; t < dims[d].tile_len; ++t) {
        if (nob < 3) obits[nob] = dims[d].start + t - dims[4].start;
        ++nob;
      }
    dims[4].len = n - dims[4].start;
    dims.resize(5);
    ok = nob <= 3;
  }
  for (const Dim& d : dims) ok = ok && d.tile_len <= 8 && d.len <= 31;  // box <= 256, extent < 2^32
  for (size_t d = 1; d < dims.size(); ++d) ok = ok && dims[d].start >= 2;  // 16-byte strides
  if (!ok) return;
  for (size_t d = 0; d < dims.size(); ++d) {
    out.tm_start[d] = dims[d].start;
    out.tm_len[d] = dims[d].len;
    out.tm_box[d] = dims[d].tile_len;
  }
  out.tm_outer = nob;
  std::copy(obits, obits + 3, out.tm_obit);
  if (re == nullptr || im == nullptr) return;  // layout only (no tensor maps)
  static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      fn = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }();
  if (!encode) return;
  cuuint64_t gdim[5], strides[4];
  cuuint32_t box[5], estr[5];
  for (size_t d = 0; d < dims.size(); ++d) {
    gdim[d] = cuuint64_t(1) << dims[d].len;
    box[d] = cuuint32_t(1) << dims[d].tile_len;
    estr[d] = 1;
    if (d > 0) strides[d - 1] = (cuuint64_t(1) << dims[d].start) * sizeof(float);
  }
  float* bases[2] = {re, im};
  bool enc_ok = true;
  for (int c = 0; c < 2 && enc_ok; ++c)
    enc_ok = encode(&out.maps[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, cuuint32_t(dims.size()), bases[c], gdim, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  if (enc_ok) out.tm_rank = uint32_t(dims.size());
}

template <int KQ>
static void launch_tc_k(const LaunchEnv& env, float* re, float* im, uint32_t n, const Sweep& s, const void* dev_mat) {
  constexpr int M2 = 1 << KQ, NCB = kTileBits - KQ;
  TcParams p{};
  p.ncb = NCB;
  int gate_rank[64], col_rank[64];
  for (int b = 0; b < 64; ++b) gate_rank[b] = col_rank[b] = -1;
  for (int j = 0; j < KQ; ++j) gate_rank[s.q[j]] = j;
  std::vector<uint32_t> tbits;
  int ncol = 0;
  for (uint32_t b = 0; b < n; ++b) {
    if (gate_rank[b] >= 0) tbits.push_back(b);
    else if (ncol < NCB) {
      col_rank[b] = ncol++;
      tbits.push_back(b);
    }
  }
  QSVB_REQUIRE(tbits.size() == size_t(kTileBits), "tc tile: state too small");
  for (int j = 0; j < 6; ++j) QSVB_REQUIRE(tbits[j] == uint32_t(j), "tc tile: low bits not contiguous");
  auto contrib = [&](uint32_t b) -> uint32_t {
    return gate_rank[b] >= 0 ? (uint32_t(1) << gate_rank[b]) << NCB : (uint32_t(1) << col_rank[b]);
  };
  uint32_t tb12[12];
  std::copy(tbits.begin(), tbits.end(), tb12);
  TileLayout lay;
  tile_layout(n, tb12, re, im, lay);
  for (int j = 0; j < 6; ++j) p.hibits[j] = lay.hibits[j];
  for (int h = 0; h < 64; ++h) {
    uint32_t d = 0;
    for (int j = 0; j < 6; ++j)
      if ((h >> j) & 1) d += contrib(p.hibits[j]);
    p.hioff[h] = lay.hioff[h];
    p.dsthi[h] = uint16_t(d);
  }
  p.runbits = lay.runbits;
  p.tm_rank = lay.tm_rank;
  p.tm_outer = lay.tm_outer;
  std::copy(lay.tm_obit, lay.tm_obit + 3, p.tm_obit);
  for (int d = 0; d < 5; ++d) {
    p.tm_start[d] = lay.tm_start[d];
    p.tm_len[d] = lay.tm_len[d];
  }
  for (int l = 0; l < 64; ++l) {
    uint32_t d = 0;
    for (int b = 0; b < 6; ++b)
      if ((l >> b) & 1) d += contrib(uint32_t(b));
    p.dstlo[l] = uint16_t(d);
  }
  // address-order tile index of each gate row / column: tile position = rank among tile bits
  auto rank_of = [&](uint32_t b) { return uint32_t(std::find(tbits.begin(), tbits.end(), b) - tbits.begin()); };
  for (int sidx = 0; sidx < M2; ++sidx) {
    uint32_t t = 0;
    for (int j = 0; j < KQ; ++j)
      if ((sidx >> j) & 1) t |= 1u << rank_of(s.q[j]);
    p.trow[sidx] = uint16_t(t);
  }
  for (int c = 0; c < (1 << NCB); ++c) {
    uint32_t t = 0;
    for (uint32_t b = 0; b < n; ++b)
      if (col_rank[b] >= 0 && ((c >> col_rank[b]) & 1)) t |= 1u << rank_of(b);
    p.tcol[c] = uint16_t(t);
    if (c < 16) {
      p.tcl[c] = stage_idx(t);
      p.tclb[c] = 4u * stage_idx(t);
    }
  }
  const bool low_cols = gate_rank[0] < 0 && gate_rank[1] < 0;
  const bool low_rows = gate_rank[0] == 0 && gate_rank[1] == 1;
  // bit 0 a column, bit 1 the gate's lowest qubit and its next qubit among state bits 2..4
  int row1_bit = -1;
  for (uint32_t b = 0; b < n; ++b)
    if (gate_rank[b] == 1) row1_bit = int(b);
  const bool lane_pair = gate_rank[0] < 0 && gate_rank[1] == 0 && row1_bit >= 2 && row1_bit <= 4;
  p.bmode = low_cols ? 0u : (low_rows ? 1u : (lane_pair ? 3u : 2u));
  p.b2_bit0 = gate_rank[0] == 0 ? 1u : 0u;
  p.pair_shift = lane_pair ? uint32_t(row1_bit - 2) : 0u;
  {
    // converter work order: float4 index bits 0..2 stay (a quarter-warp's 16-byte loads stay
    // conflict-free); for K-major tiles the lane bits 3 and 4 take the two float4 bits that make
    // the warp's B stores hit the most distinct banks (found by trying every pair)
    constexpr uint32_t CM = (1u << NCB) - 1u;
    constexpr uint32_t KRr = 2u * M2;
    auto perm_t4 = [](uint32_t u, const int (&pi)[10]) {
      uint32_t t4 = 0;
      for (int i = 0; i < 10; ++i)
        if ((u >> i) & 1u) t4 |= 1u << pi[i];
      return t4;
    };
    auto conflict = [&](const int (&pi)[10]) {
      int worst = 0;
      const int nst = p.bmode == 2 ? 2 : 1;
      for (int q = 0; q < nst; ++q) {
        int count[32] = {0};
        for (uint32_t lane = 0; lane < 32; ++lane) {
          const uint32_t t = perm_t4(lane, pi) * 4u;
          const uint32_t e = p.bmode == 2 ? (p.b2_bit0 ? 2u * q : uint32_t(q)) : 0u;
          uint32_t tl = t + e;
          if (p.bmode == 3) tl = (t & ~(4u << p.pair_shift)) | ((lane >> p.pair_shift) & 1u);
          const uint32_t d = uint32_t(p.dstlo[tl & 63u]) + p.dsthi[tl >> 6];
          const uint32_t sr = d >> NCB, c = d & CM;
          const uint32_t off = kmaj_off(c & 63u, (c >> 6) * KRr + sr, 64);
          // 4-byte stores: 32 banks per warp; 8-byte stores: 16 bank pairs per half-warp
          const uint32_t bank = p.bmode == 2 ? (off >> 2) & 31u : ((off >> 3) & 15u) + 16u * (lane >> 4);
          worst = std::max(worst, ++count[bank]);
        }
      }
      return worst;
    };
    int best[10];
    for (int i = 0; i < 10; ++i) best[i] = i;
    if (p.bmode != 0) {
      int best_c = conflict(best);
      for (int a = 3; a < 10; ++a)
        for (int b = 3; b < 10; ++b) {
          if (a == b) continue;
          int pi[10] = {0, 1, 2, a, b, 0, 0, 0, 0, 0};
          int nxt = 5;
          for (int v = 3; v < 10; ++v)
            if (v != a && v != b) pi[nxt++] = v;
          const int cc = conflict(pi);
          if (cc < best_c) {
            best_c = cc;
            std::copy(pi, pi + 10, best);
          }
        }
    }
    for (uint32_t u = 0; u < 32; ++u) {
      p.tplo[u] = uint16_t(perm_t4(u, best));
      p.tphi[u] = uint16_t(perm_t4(u << 5, best));
    }
  }

  const uint64_t ntiles = 1ull << (n - kTileBits);
  auto kern = p.bmode == 0 ? k_tc_dense<KQ, 0> : p.bmode == 1 ? k_tc_dense<KQ, 1>
             : p.bmode == 2 ? k_tc_dense<KQ, 2> : k_tc_dense<KQ, 3>;
  QSVB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTcSmem)));
  QSVB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                               int(cudaSharedmemCarveoutMaxShared)));
  // one persistent CTA per SM (the tensor-memory allocation assumes it)
  const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(env.num_sms))));
  // QSVB_TC_PROFILE=1: per-role stall cycles, averaged over CTAs, printed to stderr (synchronous)
  static const bool profile = std::getenv("QSVB_TC_PROFILE") != nullptr;
  long long* prof = nullptr;
  if (profile) QSVB_CK(cudaMalloc(&prof, sizeof(long long) * 12 * grid));
  if (prof) QSVB_CK(cudaMemsetAsync(prof, 0, sizeof(long long) * 12 * grid, env.stream));
  kern<<<grid, kTcThreads, kTcSmem, env.stream>>>(re, im, ntiles, static_cast<const uint4*>(dev_mat), p, env.err_flag,
                                                  prof, lay.maps[0], lay.maps[1]);
  QSVB_CK(cudaGetLastError());
  if (prof) {
    std::vector<long long> h(12 * size_t(grid));
    QSVB_CK(cudaMemcpyAsync(h.data(), prof, h.size() * sizeof(long long), cudaMemcpyDeviceToHost, env.stream));
    QSVB_CK(cudaStreamSynchronize(env.stream));
    cudaFree(prof);
    double avg[12] = {0};
    for (unsigned b = 0; b < grid; ++b)
      for (int k = 0; k < 12; ++k) avg[k] += double(h[12 * b + k]) / grid;
    std::fprintf(stderr,
                 "{\"tc_profile\": {\"k\": %d, \"bmode\": %u, \"tiles_per_cta\": %.1f, \"cycles\": %.0f, "
                 "\"prod_wait_empty\": %.0f, \"cvt_wait_full\": %.0f, \"cvt_wait_bfree\": %.0f, "
                 "\"mma_wait_bfull\": %.0f, \"mma_wait_dfree\": %.0f, \"epi_wait_dfull\": %.0f, "
                 "\"epi_store\": %.0f, \"epi_tmem\": %.0f, \"epi_stage\": %.0f, \"epi_sync\": %.0f}}\n",
                 KQ, p.bmode, double(ntiles) / grid, avg[7], avg[0], avg[1], avg[2], avg[3], avg[4], avg[5], avg[6],
                 avg[8], avg[9], avg[10]);
  }
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
