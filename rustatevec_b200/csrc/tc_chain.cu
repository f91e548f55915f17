// Chained tensor-core pass (complex64): up to three dense 6-qubit matrices applied, one after the
// other, to a 4096-amplitude tile that stays on the SM, then written back with a permutation of
// the tile's qubits. One read and one write of the state replace one sweep per matrix.
//
// A tile is the 2^12 amplitudes that share every state bit outside the pass's 12 tile bits (state
// bits 0..5 are always tile bits, so every global access is a contiguous run of >= 64 amplitudes).
// Matrix j acts on six tile positions (its rows) and sees the other six as 64 columns; it runs as
// the real GEMM [Yr; Yi] = W [Xr; Xi], W = [[Ur, -Ui], [Ui, Ur]] (128 x 128), with bf16 hi/lo
// split operands and an FP32 accumulator in tensor memory (Wlo Xhi + Whi Xlo + Whi Xhi), exactly
// as the single-matrix sweep (tc_dense.cu) does.
//
// One persistent CTA per SM, warp-specialised:
//   producer warp: tiled TMA or bulk copies of each tile into one of three fp32 input slots
//     (address order);
//   converter warps (8): for a tile's first matrix, split the staged fp32 tile into the bf16 hi/lo
//     B operand (one of three B buffers; layout chosen by which matrix qubits are state bits
//     0, 1); for every later matrix, gather 32 of the previous matrix's accumulator columns straight
//     from tensor memory (each warp its lane quadrant, one column per load, in the order the next
//     operand needs), split them and write them into the next B operand as 16-byte chunks of 8
//     bf16: the operand is MN- or K-major, whichever has three of its contiguous bits among the
//     previous matrix's columns (one of the two always does); chunk offsets are an XOR of a per-row
//     and a per-chunk part, both precomputed on the host; the hi/lo splits convert two values per
//     instruction (packed bf16x2);
//   MMA warps (one per B buffer; the warp walks the items on uniform control flow and one elected
//     lane issues): 24 tcgen05.mma per matrix into the tile's accumulator (64 columns), the A
//     operand (Whi, Wlo of matrix j) resident in tensor memory for the whole kernel; several items'
//     MMAs are issued concurrently;
//   epilogue warps (4): after the last matrix, read the accumulator, stage it in shared memory in
//     the permuted address order (16-byte stores when the pass's permutation puts the last matrix's
//     first two columns on output bits 0 and 1, which the planner arranges; scalar stores
//     otherwise; a per-pass XOR swizzle keeps both the staging writes and the write-back's reads
//     bank-conflict free) and write the tile back with 16-byte stores.
// Work items are (tile, matrix) pairs, walked by every role in the same order (walk_items). Up to
// two matrices, four tiles are in flight (four accumulators); three matrices leave tensor memory
// for two accumulators, so two tiles are. Either way three B buffers rotate over the items, each
// with its own MMA warp. Every mbarrier wait is bounded (a wait that runs out sets the context error flag,
// the role stops and the host reports QSVB_E_TIMEOUT). No load uses cluster multicast.
//
// k_permute_tiles applies only a tile-qubit permutation (no arithmetic): the planner uses it to put
// every qubit back on its own state bit after a run of chain passes.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>

#include "qsvb_internal.h"
#include "tc_common.cuh"

namespace qsvb {

namespace {
using namespace tc;

constexpr int kTileAmps = 4096;
constexpr int kCvtWarps = 8;
constexpr int kEpiWarps = 4;
constexpr int kCvtThreads = kCvtWarps * 32;
constexpr int kEpiThreads = kEpiWarps * 32;
constexpr int kProdWarp = kCvtWarps;       // warp 8
constexpr int kMmaWarp = kCvtWarps + 1;    // warps 9..11: the MMAs of the items of B buffer 0, 1, 2
constexpr int kMmaWarps = 3;
constexpr int kEpiWarp0 = kMmaWarp + kMmaWarps;  // warps 12..15 (lane quadrants 0..3)
constexpr int kThreads = (kEpiWarp0 + kEpiWarps) * 32;
constexpr int kTmemCols = 512;             // DEPTH accumulators (64 columns) + (Whi, Wlo) of each matrix
// Two configurations of the same kernel (template parameter DEPTH = accumulators = tiles in flight):
//   DEPTH 2 (up to three matrices): matrix j's Whi at column 128 + 128 j;
//   DEPTH 4 (one or two matrices):  matrix j's Whi at column 256 + 128 j.
// Both have 3 B buffers (one MMA warp each) and 3 input slots: 3 x 2 + 3 + 1 buffers of 32 KB with
// the output staging. With two tiles in flight the third B buffer lets the next wave's first
// conversion run while the current wave's last MMAs still read the other two.
constexpr int kBarBase = 26;               // iofull[4] ioempty[4] bfull[3] bfree[3] dfull_c[4] dfull_e[4] dfree[4]
constexpr uint32_t kBBytes = 128u * 64u * 2u;  // one of Xhi / Xlo: K = 128 rows x N = 64 bf16
constexpr uint32_t kIoBytes = kTileAmps * 8u;
constexpr int kVC = kTileAmps / 4 / kCvtThreads;   // float4 per component per converter thread
constexpr int kVE = kTileAmps / 4 / kEpiThreads;   // float4 per component per epilogue thread
constexpr size_t kChainSmem = 1024 + 3 * 2 * size_t(kBBytes) + 4 * size_t(kIoBytes) + kBarBase * 8 + 8 + 64 * 8 +
                              64 * 2 * 2 + 64 * 2 + 128 * 2;
static_assert(kChainSmem <= 232448, "chain pass: shared memory above the 227 KB per-block limit");
static_assert(kChainMaxMats * 128 + 2 * 64 <= kTmemCols && 2 * 128 + 4 * 64 <= kTmemCols, "chain pass: tensor memory");

struct ChainParams {
  // tile addressing (tile_layout)
  uint32_t hibits[6];
  uint64_t hioff[64];
  uint32_t runbits;
  uint32_t tm_rank, tm_start[5], tm_len[5], tm_outer, tm_obit[3];
  uint32_t nmat;
  // first matrix, read from the staged tile in address order: (row << 6 | column) of each value
  // of the low / high six tile positions, the converters' work order, and the B layout details
  uint16_t dstlo[64], dsthi[64];
  uint16_t tplo[32], tphi[32];
  uint32_t b2_bit0, pair_shift;
  // matrix j >= 1 read from the accumulator of matrix j - 1: the converter warp of half w gathers,
  // for chunk m (0..3) and element e (0..7), accumulator column cw[w] ^ cm[m] ^ ce[e]; the chunk's 8
  // bf16 go to B at byte offset crow[r] ^ cchunk[w][m] (+ 2 e), r = part * 64 + gate row
  uint16_t crow[kChainMaxMats][128];
  uint16_t cchunk[kChainMaxMats][2][4];
  uint8_t ce[kChainMaxMats][8], cm[kChainMaxMats][4], cw[kChainMaxMats][2];
  uint8_t bk[kChainMaxMats];  // B of matrix j >= 1 is K-major
  uint32_t evec;              // the epilogue's staging writes and reads are 16-byte vectors
  // last matrix: byte offset in the output staging of accumulator row r and of column c (XOR)
  uint16_t frow[128];
  uint16_t fcol[64];
  // the staging swizzle read by the write-back: word index of address-order position t is
  // sig_lo[t & 63] ^ sig_hi[t >> 6]
  uint16_t sig_lo[64], sig_hi[64];
};

// bf16 hi/lo split of two values, packed as bf16 pairs (the first value in the low half).
__device__ __forceinline__ void split2(uint32_t x0, uint32_t x1, uint32_t& hi, uint32_t& lo) {
  const float2 f = make_float2(__uint_as_float(x0), __uint_as_float(x1));
  const __nv_bfloat162 h = __float22bfloat162_rn(f);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __float22bfloat162_rn(make_float2(f.x - hf.x, f.y - hf.y));
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

__device__ __forceinline__ void split2f(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  split2(__float_as_uint(x0), __float_as_uint(x1), hi, lo);
}

// B layout of the first matrix (as in tc_dense.cu): 0 MN-major (state bits 0, 1 are columns),
// 1 K-major vectors (they are the matrix's rows 0, 1), 2 K-major row pairs (exactly one is a row,
// the lowest), 3 K-major vectors assembled from a lane pair (bit 0 a column, bit 1 row 0, row 1 one
// of state bits 2..4).
//
// What a converter thread does for a first matrix is the same for every tile of the pass, so it is
// worked out once (first_plan): for each of its kVC float4 groups, the staged word index t in the
// high half of plan[j] and the byte offset in B of its real parts in the low half (the imaginary
// parts follow 8192 bytes later in both layouts); layout 2 stores two pairs per group, the second
// offset in plan2[j]. Per tile, the conversion is then independent 16-byte loads, packed splits
// and stores.
template <int BM>
__device__ __forceinline__ void first_plan(const uint16_t* __restrict__ s_dlo, const uint16_t* __restrict__ s_dhi,
                                           const uint16_t* __restrict__ s_tperm, const ChainParams& p, int tid,
                                           int lane, uint32_t (&plan)[kVC], uint32_t (&plan2)[kVC]) {
  constexpr uint32_t NCB = 6, CMASK = 63;
#pragma unroll
  for (int j = 0; j < kVC; ++j) {
    const uint32_t u = uint32_t(tid + j * kCvtThreads);
    const uint32_t t = (uint32_t(s_tperm[u & 31u]) | uint32_t(s_tperm[32 + (u >> 5)])) * 4u;
    uint32_t o = 0, o2 = 0;
    if constexpr (BM == 3) {
      const uint32_t sh = p.pair_shift;
      const bool odd = ((uint32_t(lane) >> sh) & 1u) != 0;
      const uint32_t tg = (t & ~(4u << sh)) | (odd ? 1u : 0u);
      const uint32_t d = uint32_t(s_dlo[tg & 63]) + s_dhi[tg >> 6];
      o = kmaj_off(d & CMASK, d >> NCB, 64);
    } else if constexpr (BM == 2) {
      const uint32_t e1 = p.b2_bit0 ? 2u : 1u;
      const uint32_t d0 = uint32_t(s_dlo[t & 63]) + s_dhi[t >> 6];
      const uint32_t d1 = uint32_t(s_dlo[(t & 63) + e1]) + s_dhi[t >> 6];
      o = kmaj_off(d0 & CMASK, d0 >> NCB, 64);
      o2 = kmaj_off(d1 & CMASK, d1 >> NCB, 64);
    } else {
      const uint32_t d = uint32_t(s_dlo[t & 63]) + s_dhi[t >> 6];
      o = BM == 0 ? mnmaj_off(d >> NCB, d & CMASK) : kmaj_off(d & CMASK, d >> NCB, 64);
    }
    plan[j] = (t << 16) | o;
    plan2[j] = o2;
  }
}

template <int BM>
__device__ __forceinline__ void convert_first(uint32_t sre, uint32_t sim, uint32_t b_hi, uint32_t b_lo,
                                              const uint32_t (&plan)[kVC], const uint32_t (&plan2)[kVC],
                                              const ChainParams& p, int lane) {
  constexpr uint32_t kImOff = 8192;  // imaginary rows M2..2 M2-1: the second K half / 8 row groups later
  float4 xra[kVC], xia[kVC];
#pragma unroll
  for (int j = 0; j < kVC; ++j) {
    const uint32_t t4 = (plan[j] >> 16) * 4u;
    xra[j] = lds128f(sre + t4);
    xia[j] = lds128f(sim + t4);
  }
#pragma unroll
  for (int j = 0; j < kVC; ++j) {
    const float4 xr = xra[j], xi = xia[j];
    const uint32_t o = plan[j] & 0xFFFFu;
    if constexpr (BM == 3) {
      const uint32_t sh = p.pair_shift;
      const bool odd = ((uint32_t(lane) >> sh) & 1u) != 0;
      const int pm = 1 << sh;
      const float rr0 = __shfl_xor_sync(0xffffffffu, odd ? xr.x : xr.y, pm);
      const float rr1 = __shfl_xor_sync(0xffffffffu, odd ? xr.z : xr.w, pm);
      const float ri0 = __shfl_xor_sync(0xffffffffu, odd ? xi.x : xi.y, pm);
      const float ri1 = __shfl_xor_sync(0xffffffffu, odd ? xi.z : xi.w, pm);
      uint32_t h0, l0, h1, l1;
      split2f(odd ? rr0 : xr.x, odd ? rr1 : xr.z, h0, l0);
      split2f(odd ? xr.y : rr0, odd ? xr.w : rr1, h1, l1);
      sts64(b_hi + o, h0, h1);
      sts64(b_lo + o, l0, l1);
      split2f(odd ? ri0 : xi.x, odd ? ri1 : xi.z, h0, l0);
      split2f(odd ? xi.y : ri0, odd ? xi.w : ri1, h1, l1);
      sts64(b_hi + o + kImOff, h0, h1);
      sts64(b_lo + o + kImOff, l0, l1);
    } else if constexpr (BM == 2) {
      const float vr[4] = {xr.x, xr.y, xr.z, xr.w};
      const float vi[4] = {xi.x, xi.y, xi.z, xi.w};
      const int step = p.b2_bit0 ? 1 : 2;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int e = p.b2_bit0 ? 2 * q : q;
        const uint32_t oq = q == 0 ? o : plan2[j];
        uint32_t h, l;
        split2f(vr[e], vr[e + step], h, l);
        sts32(b_hi + oq, h);
        sts32(b_lo + oq, l);
        split2f(vi[e], vi[e + step], h, l);
        sts32(b_hi + oq + kImOff, h);
        sts32(b_lo + oq + kImOff, l);
      }
    } else {
      uint32_t h0, l0, h1, l1;
      split2f(xr.x, xr.y, h0, l0);
      split2f(xr.z, xr.w, h1, l1);
      sts64(b_hi + o, h0, h1);
      sts64(b_lo + o, l0, l1);
      split2f(xi.x, xi.y, h0, l0);
      split2f(xi.z, xi.w, h1, l1);
      sts64(b_hi + o + kImOff, h0, h1);
      sts64(b_lo + o + kImOff, l0, l1);
    }
  }
}

// 32 accumulator columns of this warp's 32 lanes, one column per load (addresses a[k]), all in
// flight at once, defined only once every load has completed.
__device__ __forceinline__ void tmem_ld_gather32(const uint32_t (&a)[32], uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%32];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%1}, [%33];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%2}, [%34];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%3}, [%35];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%4}, [%36];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%5}, [%37];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%6}, [%38];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%7}, [%39];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%8}, [%40];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%9}, [%41];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%10}, [%42];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%11}, [%43];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%12}, [%44];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%13}, [%45];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%14}, [%46];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%15}, [%47];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%16}, [%48];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%17}, [%49];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%18}, [%50];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%19}, [%51];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%20}, [%52];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%21}, [%53];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%22}, [%54];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%23}, [%55];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%24}, [%56];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%25}, [%57];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%26}, [%58];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%27}, [%59];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%28}, [%60];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%29}, [%61];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%30}, [%62];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%31}, [%63];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4]), "=&r"(r[5]), "=&r"(r[6]), "=&r"(r[7]), "=&r"(r[8]), "=&r"(r[9]), "=&r"(r[10]), "=&r"(r[11]), "=&r"(r[12]), "=&r"(r[13]), "=&r"(r[14]), "=&r"(r[15]), "=&r"(r[16]), "=&r"(r[17]), "=&r"(r[18]), "=&r"(r[19]), "=&r"(r[20]), "=&r"(r[21]), "=&r"(r[22]), "=&r"(r[23]), "=&r"(r[24]), "=&r"(r[25]), "=&r"(r[26]), "=&r"(r[27]), "=&r"(r[28]), "=&r"(r[29]), "=&r"(r[30]), "=&r"(r[31])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(a[8]), "r"(a[9]), "r"(a[10]), "r"(a[11]), "r"(a[12]), "r"(a[13]), "r"(a[14]), "r"(a[15]), "r"(a[16]), "r"(a[17]), "r"(a[18]), "r"(a[19]), "r"(a[20]), "r"(a[21]), "r"(a[22]), "r"(a[23]), "r"(a[24]), "r"(a[25]), "r"(a[26]), "r"(a[27]), "r"(a[28]), "r"(a[29]), "r"(a[30]), "r"(a[31])
      : "memory");
}

// Matrix j >= 1: the accumulator of matrix j - 1 (its TMEM columns from tcol, this thread's row
// offset rbase) into the B operand of matrix j, as four 16-byte chunks of hi and of lo.
__device__ __forceinline__ void convert_next(uint32_t tcol, uint32_t rbase, const uint32_t (&cc)[4],
                                             const uint32_t (&cm)[4], const uint32_t (&ce)[8],
                                             uint8_t* __restrict__ b_hi, uint8_t* __restrict__ b_lo) {
  uint32_t a[32], v[32];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int e = 0; e < 8; ++e) a[8 * m + e] = tcol + cm[m] + ce[e];
  tmem_ld_gather32(a, v);
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) split2(v[8 * m + 2 * i], v[8 * m + 2 * i + 1], h[i], l[i]);
    const uint32_t off = rbase ^ cc[m];
    const uint32_t sh = smem_u32(b_hi + off), sl = smem_u32(b_lo + off);
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sh), "r"(h[0]), "r"(h[1]), "r"(h[2]), "r"(h[3])
                 : "memory");
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sl), "r"(l[0]), "r"(l[1]), "r"(l[2]), "r"(l[3])
                 : "memory");
  }
}

// The order in which every role walks the work items (tile k, matrix j). Item i uses B buffer
// i % NB and accumulator k % DEPTH.
//   DEPTH 2: waves of two tiles: matrix 0 of both, then matrix 1 of both, ... (the MMA of one tile
//     overlaps the conversion of the other);
//   DEPTH 4: a skewed stream: step s holds matrix 0 of tile s, then matrix 1 of tile s - 2, so two
//     other conversions separate a tile's two conversions (covering its first MMA) and the staged
//     tiles are consumed one per two items, evenly.
// Every item depends only on earlier items of the same walk (its previous matrix, its B buffer's
// previous item, the tile that last held its accumulator), so the pipeline cannot deadlock.
// f(k, j, i) returns false to stop the walk.
template <int DEPTH, class F>
__device__ __forceinline__ void walk_items(uint32_t ntiles, uint32_t nmat, F&& f) {
  uint32_t i = 0;
  if constexpr (DEPTH == 2) {
    for (uint32_t w0 = 0; w0 < ntiles; w0 += 2) {
      const uint32_t nt = ntiles - w0 < 2u ? ntiles - w0 : 2u;
      for (uint32_t j = 0; j < nmat; ++j)
        for (uint32_t tt = 0; tt < nt; ++tt, ++i)
          if (!f(w0 + tt, j, i)) return;
    }
  } else {
    constexpr uint32_t L = 2;
    const uint32_t steps = ntiles + (nmat - 1) * L;
    for (uint32_t st = 0; st < steps; ++st)
      for (uint32_t j = 0; j < nmat; ++j) {
        if (st < j * L || st - j * L >= ntiles) continue;
        if (!f(st - j * L, j, i)) return;
        ++i;
      }
  }
}

template <int BM, int DEPTH>
__global__ void __launch_bounds__(kThreads, 1) k_tc_chain(float* __restrict__ re, float* __restrict__ im,
                                                          uint64_t ntiles, const uint4* __restrict__ wpack,
                                                          const __grid_constant__ ChainParams p, int* err,
                                                          const __grid_constant__ CUtensorMap tm_re,
                                                          const __grid_constant__ CUtensorMap tm_im) {
  constexpr int NB = 3;                        // B buffers (one MMA warp each)
  constexpr int NIO = 3;                       // input slots
  constexpr uint32_t A0 = 64u * DEPTH;         // tensor-memory column of matrix 0's Whi
  static_assert(A0 + 128u * (DEPTH == 2 ? 3u : 2u) <= uint32_t(kTmemCols), "chain pass: tensor memory");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* bbuf = smem;                                               // buffer b: hi, then lo
  float* io = reinterpret_cast<float*>(bbuf + NB * 2 * kBBytes);      // slot s: re [4096], im [4096]
  float* ostage = io + NIO * 2 * kTileAmps;                           // the epilogue's result
  uint64_t* bars = reinterpret_cast<uint64_t*>(ostage + 2 * kTileAmps);
  uint64_t* iofull = bars;        // [NIO] TMA complete_tx -> converters
  uint64_t* ioempty = bars + 4;   // [NIO] converters -> producer
  uint64_t* bfull = bars + 8;     // [NB] converters -> MMA
  uint64_t* bfree = bars + 11;    // [NB] MMA commit -> converters
  // accumulators: each barrier has one consumer role that waits on every one of its phases in
  // order (a parity wait cannot tell a completion from the one two phases later, so no role may
  // skip phases that belong to another)
  uint64_t* dfull_c = bars + 14;  // [DEPTH] MMA commit -> converters (accumulators of matrices 0..nmat-2)
  uint64_t* dfull_e = bars + 18;  // [DEPTH] MMA commit -> epilogue (accumulators of the last matrix)
  uint64_t* dfree = bars + 22;    // [DEPTH] accumulator read -> MMA
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + kBarBase);
  uint64_t* s_hioff = reinterpret_cast<uint64_t*>(bars + kBarBase + 1);
  uint16_t* s_dlo = reinterpret_cast<uint16_t*>(s_hioff + 64);
  uint16_t* s_dhi = s_dlo + 64;
  uint16_t* s_tperm = s_dhi + 64;   // tplo [32], tphi [32]
  uint16_t* s_sig = s_tperm + 64;   // sig_lo [64], sig_hi [64]

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t nmat = p.nmat;
  for (int i = tid; i < 64; i += kThreads) {
    s_hioff[i] = p.hioff[i];
    s_dlo[i] = p.dstlo[i];
    s_dhi[i] = p.dsthi[i];
    s_sig[i] = p.sig_lo[i];
    s_sig[64 + i] = p.sig_hi[i];
  }
  for (int i = tid; i < 32; i += kThreads) {
    s_tperm[i] = p.tplo[i];
    s_tperm[32 + i] = p.tphi[i];
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    // converter and epilogue barriers take one arrival per warp (lane 0, after the warp's lanes
    // have synchronised): 256 single-thread arrivals on one barrier word serialise for hundreds of
    // cycles
    for (int s = 0; s < NIO; ++s) {
      mbar_init(&iofull[s], 1);
      mbar_init(&ioempty[s], kCvtWarps);
    }
    for (int s = 0; s < NB; ++s) {
      mbar_init(&bfull[s], kCvtWarps);
      mbar_init(&bfree[s], 1);
    }
    for (int s = 0; s < DEPTH; ++s) {
      mbar_init(&dfull_c[s], 1);
      mbar_init(&dfull_e[s], 1);
      // every converter warp (count 1) or every epilogue warp (count 2) once it has read the
      // accumulator
      mbar_init(&dfree[s], kCvtWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  if (warp >= kEpiWarp0) {
    // A (Whi, Wlo of every matrix) into tensor memory: lane m holds row m, 64 32-bit columns of
    // packed bf16 pairs (element 2j in the low half)
    const uint32_t quad = uint32_t(warp & 3), m = quad * 32 + uint32_t(lane);
    for (uint32_t j = 0; j < nmat; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        uint32_t r[64];
        const uint4* src = wpack + ((size_t(j) * 2 + size_t(h)) * 128 + m) * 16;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const uint4 u = src[q];
          r[4 * q] = u.x;
          r[4 * q + 1] = u.y;
          r[4 * q + 2] = u.z;
          r[4 * q + 3] = u.w;
        }
        tmem_st64(tmem + ((quad * 32) << 16) + A0 + 128u * j + 64u * uint32_t(h), r);
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
  uint32_t my_tiles =  // this CTA's tiles (a role whose checked tables fail sets it to 0)
      uint64_t(blockIdx.x) < ntiles ? uint32_t((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0u;

  if (warp == kProdWarp) {
    // ============================ producer: the tile's runs into an input slot (address order)
    const uint32_t rb = p.runbits, nruns = uint32_t(kTileAmps) >> rb, run_bytes = 4u << rb;
    for (uint32_t i = 0; i < my_tiles; ++i) {
      const uint32_t slot = i % NIO, par = (i / NIO) & 1u;
      bool ok = true;
      if (lane == 0) {
        ok = mbar_wait(&ioempty[slot], par ^ 1u);
        if (ok) mbar_arrive_expect_tx(&iofull[slot], kIoBytes);
        else atomicOr(err, kErrTimeout);
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
      const uint64_t base = tile_base(blockIdx.x + uint64_t(i) * gridDim.x);
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
    // ============================ converters: B operand of every (tile, matrix) item
    const uint32_t quad = uint32_t(warp & 3), half = uint32_t(warp >> 2);
    const uint32_t row = quad * 32 + uint32_t(lane);  // accumulator row this thread reads
    uint32_t rb1 = 0, rb2 = 0;                        // its byte offsets in the B of matrices 1 and 2
    if (nmat > 1) rb1 = p.crow[1][row];
    if (nmat > 2) rb2 = p.crow[2][row];
    const uint32_t lane_base = tmem + ((quad * 32) << 16);
    uint32_t plan[kVC], plan2[kVC];
    first_plan<BM>(s_dlo, s_dhi, s_tperm, p, tid, lane, plan, plan2);
    // (checked builds) every staged word, operand offset and accumulator column this thread will
    // use, once: a converter warp whose tables fail stops, and the pass ends through its bounded
    // waits
    bool tables_ok = true;
#pragma unroll
    for (int v = 0; v < kVC; ++v)
      tables_ok = tables_ok && QSVB_BC((plan[v] >> 16) + 4 <= uint32_t(kTileAmps) &&
                                           (plan[v] & 0xFFFFu) + 8192u + (BM == 2 ? 4u : 8u) <= kBBytes &&
                                           (BM != 2 || plan2[v] + 8192u + 4u <= kBBytes),
                                       err);
    for (uint32_t j = 1; j < nmat; ++j)
      for (int m = 0; m < 4; ++m) {
        tables_ok = tables_ok && QSVB_BC(((j == 1 ? rb1 : rb2) ^ p.cchunk[j][half][m]) + 16u <= kBBytes, err);
        for (int e = 0; e < 8; ++e)
          tables_ok = tables_ok && QSVB_BC(uint32_t(p.cw[j][half]) + p.cm[j][m] + p.ce[j][e] < 64u, err);
      }
    if (!__all_sync(0xffffffffu, tables_ok)) my_tiles = 0;
    uint32_t cpar = 0;  // bit a: parity of the intermediate accumulators of slot a consumed so far
    walk_items<DEPTH>(my_tiles, nmat, [&](uint32_t k, uint32_t j, uint32_t i) -> bool {
      const uint32_t slot = k % NIO, bs = i % NB, bpar = (i / NB) & 1u, a = k % DEPTH;
      // the input: the staged tile (matrix 0) or the accumulator of this tile's previous matrix;
      // the converters consume every intermediate accumulator, slot by slot in item order. Lane 0
      // waits for the warp (a barrier polled by all 32 lanes costs hundreds of cycles); the warp
      // synchronisation after it orders the other lanes' reads after its acquire.
      bool ready = true;
      if (lane == 0) {
        ready = j == 0 ? mbar_wait(&iofull[slot], (k / NIO) & 1u) : mbar_wait(&dfull_c[a], (cpar >> a) & 1u);
        ready = ready && mbar_wait(&bfree[bs], bpar ^ 1u);
      }
      if (j > 0) cpar ^= 1u << a;
      ready = __shfl_sync(0xffffffffu, ready ? 1 : 0, 0) != 0;
      __syncwarp();
      if (!ready) {
        atomicOr(err, kErrTimeout);
        return false;
      }
      uint8_t* b_hi = bbuf + bs * 2 * kBBytes;
      uint8_t* b_lo = b_hi + kBBytes;
      if (j == 0) {
        const uint32_t sre = smem_u32(io + slot * 2 * kTileAmps);
        convert_first<BM>(sre, sre + kTileAmps * 4u, smem_u32(b_hi), smem_u32(b_lo), plan, plan2, p, lane);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // B writes -> the MMA's reads
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&bfull[bs]);
          mbar_arrive(&ioempty[slot]);  // the staged tile has been read
        }
      } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t cc[4], cmv[4], cev[8];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          cc[m] = p.cchunk[j][half][m];
          cmv[m] = p.cm[j][m];
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) cev[e] = p.ce[j][e];
        convert_next(lane_base + a * 64u + p.cw[j][half], j == 1 ? rb1 : rb2, cc, cmv, cev, b_hi, b_lo);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&dfree[a]);  // the warp's part of the accumulator has been read
          mbar_arrive(&bfull[bs]);
        }
      }
      return true;
    });
  } else if (warp < kMmaWarp + kMmaWarps) {
    // ============================ MMA issue: the items of one B buffer; the whole warp walks them
    // (uniform operands), one elected lane issues
    const uint32_t own = uint32_t(warp - kMmaWarp);
    if (own < uint32_t(NB)) {
      const uint32_t leader = elect_one();
      // idesc: f32 accumulate, bf16 A and B, K-major A; B MN-major (bit 16) for every matrix but
      // a K-major first one; N = 64, M = 128
      const uint32_t idesc_k =
          (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(64 >> 3) << 17) | (uint32_t(128 >> 4) << 24);
      const uint32_t idesc_mn = idesc_k | (1u << 16);
      uint32_t upar = 0;  // bit a: parity of the MMAs into accumulator a so far (all warps' items)
      walk_items<DEPTH>(my_tiles, nmat, [&](uint32_t k, uint32_t j, uint32_t i) -> bool {
        const uint32_t a = k % DEPTH, u = (upar >> a) & 1u;
        upar ^= 1u << a;
        const uint32_t bs = i % NB;
        if (bs != own) return true;
        // the accumulator's previous content (consumed before this MMA can be issued, so the
        // wait cannot see a phase two ahead)
        const bool ok = mbar_wait(&bfull[bs], (i / NB) & 1u) && mbar_wait(&dfree[a], u ^ 1u);
        if (!__all_sync(0xffffffffu, ok)) {
          if (leader) atomicOr(err, kErrTimeout);
          return false;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const bool mn = j > 0 ? p.bk[j] == 0 : BM == 0;
        const uint32_t d_tmem = tmem + a * 64u;
        const uint32_t a_hi = tmem + A0 + 128u * j, a_lo = a_hi + 64u;
        // descriptors of K step 0; step s adds its byte offset (>> 4) to the address field
        const uint64_t dbh0 = sw128_desc(smem_u32(bbuf + bs * 2 * kBBytes), mn ? 128u * 128u : 16u, 1024u);
        const uint64_t dbl0 = dbh0 + (kBBytes >> 4);
        if (mn) {
#pragma unroll
          for (int s = 0; s < 8; ++s) {
            const uint64_t o = uint64_t(s) * (2048u >> 4);
            mma_bf16_ts_by(leader, d_tmem, a_lo + uint32_t(s) * 8u, dbh0 + o, idesc_mn, s > 0 ? 1u : 0u);
            mma_bf16_ts_by(leader, d_tmem, a_hi + uint32_t(s) * 8u, dbl0 + o, idesc_mn, 1u);
            mma_bf16_ts_by(leader, d_tmem, a_hi + uint32_t(s) * 8u, dbh0 + o, idesc_mn, 1u);
          }
        } else {
#pragma unroll
          for (int s = 0; s < 8; ++s) {
            const uint64_t o = uint64_t((s >> 2) * (64 * 128) + (s & 3) * 32) >> 4;
            mma_bf16_ts_by(leader, d_tmem, a_lo + uint32_t(s) * 8u, dbh0 + o, idesc_k, s > 0 ? 1u : 0u);
            mma_bf16_ts_by(leader, d_tmem, a_hi + uint32_t(s) * 8u, dbl0 + o, idesc_k, 1u);
            mma_bf16_ts_by(leader, d_tmem, a_hi + uint32_t(s) * 8u, dbh0 + o, idesc_k, 1u);
          }
        }
        mma_commit_by(leader, &bfree[bs]);  // B buffer consumed
        mma_commit_by(leader, j + 1 < nmat ? &dfull_c[a] : &dfull_e[a]);  // accumulator ready for its consumer
        return true;
      });
    }
    __syncwarp();
  } else {
    // ============================ epilogue: last matrix's accumulator -> staging -> global
    const int quad = warp & 3;
    const int et = tid - kEpiWarp0 * 32;
    const uint32_t row = uint32_t(quad * 32 + lane);
    const uint32_t frow = p.frow[row];
    const bool evec = p.evec != 0;
    bool tables_ok = true;  // (checked builds) the staging offsets of this thread's row, once
    for (int q = 0; q < 64; q += evec ? 4 : 1)
      tables_ok = tables_ok && QSVB_BC((frow ^ uint32_t(p.fcol[q])) + (evec ? 16u : 4u) <= 2u * kTileAmps * 4u, err);
    if (!named_all(3, kEpiThreads, tables_ok)) my_tiles = 0;
    uint32_t epar = 0;  // bit a: parity of the final accumulators of slot a consumed so far
    walk_items<DEPTH>(my_tiles, nmat, [&](uint32_t k, uint32_t j, uint32_t) -> bool {
      if (j + 1 != nmat) return true;  // items of the earlier matrices belong to the converters
      const uint32_t a = k % DEPTH;
      const bool ready = lane != 0 || mbar_wait(&dfull_e[a], (epar >> a) & 1u);  // lane 0 waits for the warp
      epar ^= 1u << a;
      // one decision for all epilogue threads (the barrier also orders every lane after its warp's
      // acquire); reaching it also means every thread's reads of the previous tile's staging are done
      if (!named_all(2, kEpiThreads, ready)) {
        atomicOr(err, kErrTimeout);
        return false;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t v[64];
      tmem_ld64_wait(tmem + (uint32_t(quad * 32) << 16) + a * 64u, v);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive_cnt(&dfree[a], 2);  // 4 epilogue warps stand for the 8 converter warps
      const uint32_t st = smem_u32(ostage);
      if (evec) {
        // columns 4k..4k+3 are four consecutive output positions: one 16-byte store each
#pragma unroll
        for (int q = 0; q < 16; ++q)
          sts128f(st + (frow ^ uint32_t(p.fcol[4 * q])),
                  make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]), __uint_as_float(v[4 * q + 2]),
                              __uint_as_float(v[4 * q + 3])));
      } else {
#pragma unroll
        for (int q = 0; q < 64; ++q) sts32(st + (frow ^ uint32_t(p.fcol[q])), v[q]);
      }
      named_sync(1, kEpiThreads);  // the whole result is staged
      const uint64_t base = tile_base(blockIdx.x + uint64_t(k) * gridDim.x);
      const uint32_t s1 = p.sig_lo[1], s2 = p.sig_lo[2], s3 = p.sig_lo[3];
#pragma unroll
      for (int q = 0; q < kVE; ++q) {
        const int t = (et + q * kEpiThreads) * 4, tlo = t & 63, thi = t >> 6;
        const uint64_t ad = base + s_hioff[thi] + uint64_t(tlo);
        const uint32_t w = uint32_t(s_sig[tlo]) ^ s_sig[64 + thi];
        if (!QSVB_BC((evec ? w + 4 <= uint32_t(kTileAmps) : w < uint32_t(kTileAmps)) && ad + 4 <= (ntiles << 12), err))
          continue;
        float4 xr, xi;
        if (evec) {  // the swizzle keeps bits 0, 1: positions t..t+3 are words w..w+3
          xr = lds128f(st + w * 4u);
          xi = lds128f(st + (kTileAmps + w) * 4u);
        } else {
          xr.x = ostage[w];
          xr.y = ostage[w ^ s1];
          xr.z = ostage[w ^ s2];
          xr.w = ostage[w ^ s3];
          xi.x = ostage[kTileAmps + w];
          xi.y = ostage[kTileAmps + (w ^ s1)];
          xi.z = ostage[kTileAmps + (w ^ s2)];
          xi.w = ostage[kTileAmps + (w ^ s3)];
        }
        __stcs(reinterpret_cast<float4*>(re + ad), xr);
        __stcs(reinterpret_cast<float4*>(im + ad), xi);
      }
      return true;
    });
  }
  __syncwarp();  // roles may leave their loops at different iterations after a timeout
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

// ---------------------------------------------------------------- tile permutation (no arithmetic)
constexpr int kPermThreads = 256;

struct PermParams {
  uint32_t hibits[6];
  uint64_t hioff[64];
  uint16_t plo[64], phi[64];  // destination tile position of each value of the low / high six bits
};

// Each block moves its tiles through shared memory: 16-byte loads of the tile in address order,
// scalar stores at the permuted positions, 16-byte stores back to the same tile's addresses (the
// set of addresses a tile covers is closed under its permutation, so the update is in place).
template <class R>
__global__ void __launch_bounds__(kPermThreads) k_permute_tiles(R* __restrict__ re, R* __restrict__ im, uint64_t ntiles,
                                                                const __grid_constant__ PermParams p) {
  using V = typename std::conditional<sizeof(R) == 4, float4, double2>::type;
  constexpr int VN = 16 / sizeof(R);  // amplitudes per 16-byte vector
  extern __shared__ __align__(16) uint8_t smem_raw[];
  R* sre = reinterpret_cast<R*>(smem_raw);
  R* sim = sre + kTileAmps;
  __shared__ uint64_t s_hioff[64];
  __shared__ uint16_t s_plo[64], s_phi[64];
  for (int i = threadIdx.x; i < 64; i += kPermThreads) {
    s_hioff[i] = p.hioff[i];
    s_plo[i] = p.plo[i];
    s_phi[i] = p.phi[i];
  }
  __syncthreads();
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    uint64_t base = tile << 6;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const uint32_t b = p.hibits[j];
      const uint64_t lo = base & ((1ull << b) - 1ull);
      base = ((base - lo) << 1) | lo;
    }
    for (int u = threadIdx.x; u < kTileAmps / VN; u += kPermThreads) {
      const int t = u * VN, tlo = t & 63, thi = t >> 6;
      const uint64_t a = base + s_hioff[thi] + uint64_t(tlo);
      const V xr = *reinterpret_cast<const V*>(re + a);
      const V xi = *reinterpret_cast<const V*>(im + a);
      const R* vr = reinterpret_cast<const R*>(&xr);
      const R* vi = reinterpret_cast<const R*>(&xi);
      const uint32_t dhi = s_phi[thi];
#pragma unroll
      for (int e = 0; e < VN; ++e) {
        const uint32_t d = dhi ^ s_plo[tlo + e];
        sre[d] = vr[e];
        sim[d] = vi[e];
      }
    }
    __syncthreads();
    for (int u = threadIdx.x; u < kTileAmps / VN; u += kPermThreads) {
      const int t = u * VN, tlo = t & 63, thi = t >> 6;
      const uint64_t a = base + s_hioff[thi] + uint64_t(tlo);
      *reinterpret_cast<V*>(re + a) = *reinterpret_cast<const V*>(sre + t);
      *reinterpret_cast<V*>(im + a) = *reinterpret_cast<const V*>(sim + t);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- host-side tables
uint32_t deposit6(uint32_t v, const uint8_t (&pos)[6]) {
  uint32_t t = 0;
  for (int i = 0; i < 6; ++i)
    if ((v >> i) & 1u) t |= 1u << pos[i];
  return t;
}
uint32_t gather6(uint32_t t, const uint8_t (&pos)[6]) {
  uint32_t v = 0;
  for (int i = 0; i < 6; ++i) v |= ((t >> pos[i]) & 1u) << i;
  return v;
}
uint32_t permute12(uint32_t t, const uint8_t (&perm)[12]) {
  uint32_t o = 0;
  for (int i = 0; i < 12; ++i)
    if ((t >> i) & 1u) o |= 1u << perm[i];
  return o;
}
int rank5(std::vector<uint32_t> v) {  // GF(2) rank of 5-bit vectors
  int r = 0;
  for (int bit = 4; bit >= 0; --bit) {
    size_t piv = v.size();
    for (size_t i = size_t(r); i < v.size(); ++i)
      if ((v[i] >> bit) & 1u) {
        piv = i;
        break;
      }
    if (piv == v.size()) continue;
    std::swap(v[size_t(r)], v[piv]);
    for (size_t i = 0; i < v.size(); ++i)
      if (i != size_t(r) && ((v[i] >> bit) & 1u)) v[i] ^= v[size_t(r)];
    ++r;
  }
  return r;
}

// The output staging swizzle: word index of position t = t ^ A(t >> 5), A a 7-bit -> 5-bit GF(2)
// map (bits 5..11 stay, so it is a bijection). Scalar epilogue: the epilogue's 32 lanes (positions
// lane_pos[0..4] for lane bits 0..4) and the write-back's 32 lanes (position bits 2..6) each hit 32
// distinct banks. Vector epilogue (16-byte accesses, served 8 lanes at a time): A leaves bits 0, 1
// alone, and the 8 lanes of each phase (lane bits 0..2) hit 8 distinct 16-byte bank groups in both
// accesses. Deterministic search; A = 0 (correct, with bank conflicts) if none is found.
void staging_swizzle(const uint32_t (&lane_pos)[5], bool vec, uint16_t (&sig_lo)[64], uint16_t (&sig_hi)[64]) {
  uint32_t A[7] = {0, 0, 0, 0, 0, 0, 0};
  auto word_of_bit = [&](uint32_t pos, const uint32_t (&a)[7]) { return pos < 5 ? (1u << pos) : a[pos - 5]; };
  uint64_t rng = 0x9E3779B97F4A7C15ull;
  for (int attempt = 0; attempt < 20000; ++attempt) {
    uint32_t a[7];
    for (int i = 0; i < 7; ++i) {
      rng ^= rng << 13;
      rng ^= rng >> 7;
      rng ^= rng << 17;
      a[i] = vec ? (uint32_t(rng) & 7u) << 2 : uint32_t(rng) & 31u;
    }
    if (attempt == 0) std::fill(a, a + 7, 0u);
    bool ok;
    if (vec) {
      std::vector<uint32_t> e;
      for (int b = 0; b < 3; ++b) e.push_back(word_of_bit(lane_pos[b], a) >> 2);
      ok = rank5(e) == 3;  // the write-back's phases vary bits 2..4 of t only: always distinct
    } else {
      std::vector<uint32_t> w = {word_of_bit(2, a), word_of_bit(3, a), word_of_bit(4, a), word_of_bit(5, a),
                                 word_of_bit(6, a)};
      std::vector<uint32_t> e;
      for (uint32_t b : lane_pos) e.push_back(word_of_bit(b, a));
      ok = rank5(w) == 5 && rank5(e) == 5;
    }
    if (ok) {
      std::copy(a, a + 7, A);
      break;
    }
  }
  auto sig = [&](uint32_t t) {
    uint32_t w = t;
    for (int i = 0; i < 7; ++i)
      if ((t >> (5 + i)) & 1u) w ^= A[i];
    return w;
  };
  for (uint32_t i = 0; i < 64; ++i) {
    sig_lo[i] = uint16_t(sig(i));
    sig_hi[i] = uint16_t(sig(i << 6));
  }
}

// Layout class of the first matrix's B operand (the bmode of convert_first) from its rows.
uint32_t first_bmode(const uint8_t (&rows0)[6], uint32_t* b2_bit0 = nullptr, uint32_t* pair_shift = nullptr) {
  int rank0[12];
  for (int t = 0; t < 12; ++t) rank0[t] = -1;
  for (int i = 0; i < 6; ++i) rank0[rows0[i]] = i;
  int row1_pos = -1;
  for (int t = 0; t < 12; ++t)
    if (rank0[t] == 1) row1_pos = t;
  const bool low_cols = rank0[0] < 0 && rank0[1] < 0;
  const bool low_rows = rank0[0] == 0 && rank0[1] == 1;
  const bool lane_pair = rank0[0] < 0 && rank0[1] == 0 && row1_pos >= 2 && row1_pos <= 4;
  if (b2_bit0) *b2_bit0 = rank0[0] == 0 ? 1u : 0u;
  if (pair_shift) *pair_shift = lane_pair ? uint32_t(row1_pos - 2) : 0u;
  return low_cols ? 0u : (low_rows ? 1u : (lane_pair ? 3u : 2u));
}

// Byte offset of element (kk, n) in a B operand of 128 K-rows x 64 columns, MN- or K-major (both
// XOR-linear in the bits of kk and n).
uint32_t b_off(bool kmajor, uint32_t kk, uint32_t n) { return kmajor ? kmaj_off(n, kk, 64) : mnmaj_off(kk, n); }

bool contains6(const uint8_t (&a)[6], uint8_t v) { return std::find(a, a + 6, v) != a + 6; }
int index6(const uint8_t (&a)[6], uint8_t v) { return int(std::find(a, a + 6, v) - a); }

// Every table entry the kernel indexes shared memory with stays inside its buffer and maps its
// domain one to one (a violated check is a planner or table bug, reported before any launch).
void check_chain_params(const ChainParams& p, uint32_t nm) {
  std::vector<char> seen(size_t(1) << 15);
  auto reset = [&] { std::fill(seen.begin(), seen.end(), 0); };
  reset();
  for (uint32_t h = 0; h < 64; ++h)
    for (uint32_t l = 0; l < 64; ++l) {
      const uint32_t d = uint32_t(p.dstlo[l]) ^ p.dsthi[h];
      QSVB_REQUIRE(d < 4096 && !seen[d], "chain pass: first-matrix index table is not a bijection");
      seen[d] = 1;
    }
  for (uint32_t j = 1; j < nm; ++j) {
    reset();
    std::vector<char> col_seen(64, 0);
    for (uint32_t w = 0; w < 2; ++w)
      for (uint32_t m = 0; m < 4; ++m)
        for (uint32_t e = 0; e < 8; ++e) {
          const uint32_t c = uint32_t(p.cw[j][w]) ^ p.cm[j][m] ^ p.ce[j][e];
          QSVB_REQUIRE(c < 64 && !col_seen[c], "chain pass: accumulator column gather is not a bijection");
          col_seen[c] = 1;
          for (uint32_t r = 0; r < 128; ++r) {
            const uint32_t chunk = uint32_t(p.crow[j][r]) ^ p.cchunk[j][w][m];
            QSVB_REQUIRE((chunk & 15u) == 0, "chain pass: operand chunk not 16-byte aligned");
            const uint32_t o = chunk + 2 * e;
            QSVB_REQUIRE(o < kBBytes && !seen[o], "chain pass: operand scatter table out of range");
            seen[o] = 1;
          }
        }
  }
  reset();
  for (uint32_t r = 0; r < 128; ++r)
    for (uint32_t c = 0; c < 64; ++c) {
      const uint32_t o = uint32_t(p.frow[r]) ^ p.fcol[c];
      QSVB_REQUIRE(o < 2u * kTileAmps * 4u && (o & 3u) == 0 && !seen[o >> 2],
                   "chain pass: output staging table out of range");
      seen[o >> 2] = 1;
      if (p.evec && (c & 3u))
        QSVB_REQUIRE(o == ((uint32_t(p.frow[r]) ^ p.fcol[c & ~3u]) + 4u * (c & 3u)),
                     "chain pass: vector epilogue columns are not consecutive outputs");
    }
  reset();
  for (uint32_t h = 0; h < 64; ++h)
    for (uint32_t l = 0; l < 64; ++l) {
      const uint32_t w = uint32_t(p.sig_lo[l]) ^ p.sig_hi[h];
      QSVB_REQUIRE(w < 4096 && !seen[w], "chain pass: staging swizzle is not a bijection");
      QSVB_REQUIRE(!p.evec || (w & 3u) == (l & 3u), "chain pass: vector staging swizzle moves bits 0, 1");
      seen[w] = 1;
    }
  reset();
  for (uint32_t u = 0; u < 1024; ++u) {
    const uint32_t t4 = uint32_t(p.tplo[u & 31u]) | p.tphi[u >> 5];
    QSVB_REQUIRE(t4 < 1024 && !seen[t4], "chain pass: converter work order is not a permutation");
    seen[t4] = 1;
  }
}

// The kernel's parameter tables for one chain pass (tile addressing, operand gathers and chunk
// offsets, output staging), checked to stay inside their buffers; returns the first matrix's B
// layout mode.
uint32_t build_chain_params(const Sweep& s, uint32_t n, float* re, float* im, ChainParams& p, TileLayout& lay) {
  QSVB_REQUIRE(n >= 12, "chain pass: state too small");
  QSVB_REQUIRE(s.chain_nmat >= 1 && s.chain_nmat <= uint32_t(kChainMaxMats), "chain pass: 1..3 matrices");
  const uint32_t nm = s.chain_nmat;
  std::memset(&p, 0, sizeof(p));
  p.nmat = nm;
  tile_layout(n, s.chain_tbits, re, im, lay);
  std::copy(lay.hibits, lay.hibits + 6, p.hibits);
  std::copy(lay.hioff, lay.hioff + 64, p.hioff);
  p.runbits = lay.runbits;
  p.tm_rank = lay.tm_rank;
  std::copy(lay.tm_start, lay.tm_start + 5, p.tm_start);
  std::copy(lay.tm_len, lay.tm_len + 5, p.tm_len);
  p.tm_outer = lay.tm_outer;
  std::copy(lay.tm_obit, lay.tm_obit + 3, p.tm_obit);
  uint8_t rows[kChainMaxMats][6], cols[kChainMaxMats][6];
  for (uint32_t j = 0; j < nm; ++j) {
    std::copy(s.chain_rows[j], s.chain_rows[j] + 6, rows[j]);
    std::copy(s.chain_cols[j], s.chain_cols[j] + 6, cols[j]);
    uint32_t all = 0;
    for (int i = 0; i < 6; ++i) all |= (1u << rows[j][i]) | (1u << cols[j][i]);
    QSVB_REQUIRE(all == 0xFFFu, "chain pass: rows and columns must cover the 12 tile positions");
  }
  // first matrix, read in address order: rows ascend (the B layout modes rely on the lowest rows),
  // and with bit 0 and 1 both columns (MN-major vectors) they are its columns 0 and 1
  bool rows_ascending = true;
  for (int i = 1; i < 6; ++i) rows_ascending = rows_ascending && rows[0][i] > rows[0][i - 1];
  QSVB_REQUIRE(rows_ascending, "chain pass: the first matrix's rows must ascend");
  const uint32_t bmode = first_bmode(rows[0], &p.b2_bit0, &p.pair_shift);
  QSVB_REQUIRE(bmode != 0 || (cols[0][0] == 0 && cols[0][1] == 1),
               "chain pass: state bits 0, 1 must be the first matrix's columns 0, 1");
  auto d_of = [&](uint32_t j, uint32_t t) { return (gather6(t, rows[j]) << 6) | gather6(t, cols[j]); };
  for (uint32_t l = 0; l < 64; ++l) {
    p.dstlo[l] = uint16_t(d_of(0, l));
    p.dsthi[l] = uint16_t(d_of(0, l << 6));
  }
  {
    // converter work order (as in tc_dense.cu): float4 index bits 0..2 stay; for K-major layouts the
    // lane bits 3 and 4 take the two float4 bits that spread the warp's B stores over most banks
    auto perm_t4 = [](uint32_t u, const int (&pi)[10]) {
      uint32_t t4 = 0;
      for (int i = 0; i < 10; ++i)
        if ((u >> i) & 1u) t4 |= 1u << pi[i];
      return t4;
    };
    auto conflict = [&](const int (&pi)[10]) {
      int worst = 0;
      const int nst = bmode == 2 ? 2 : 1;
      for (int q = 0; q < nst; ++q) {
        int count[32] = {0};
        for (uint32_t ln = 0; ln < 32; ++ln) {
          const uint32_t t = perm_t4(ln, pi) * 4u;
          const uint32_t e = bmode == 2 ? (p.b2_bit0 ? 2u * q : uint32_t(q)) : 0u;
          uint32_t tl = t + e;
          if (bmode == 3) tl = (t & ~(4u << p.pair_shift)) | ((ln >> p.pair_shift) & 1u);
          const uint32_t d = uint32_t(p.dstlo[tl & 63u]) + p.dsthi[tl >> 6];
          const uint32_t off = kmaj_off(d & 63u, d >> 6, 64);
          const uint32_t bank = bmode == 2 ? (off >> 2) & 31u : ((off >> 3) & 15u) + 16u * (ln >> 4);
          worst = std::max(worst, ++count[bank]);
        }
      }
      return worst;
    };
    int best[10];
    for (int i = 0; i < 10; ++i) best[i] = i;
    if (bmode != 0) {
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
  // later matrices: the accumulator of matrix j - 1 into the B of matrix j. The B layout's three
  // contiguous bits (column slots 0..2 when MN-major, row slots 0..2 when K-major) are columns of
  // matrix j - 1: each converter thread gathers, per 16-byte chunk, the 8 accumulator columns that
  // differ only in those three bits; the half of the columns a warp takes is fixed by one other
  // column bit, and the chunk by the remaining two.
  auto pos_of = [&](uint32_t j, uint32_t srow, uint32_t col) { return deposit6(srow, rows[j]) | deposit6(col, cols[j]); };
  for (uint32_t j = 1; j < nm; ++j) {
    const bool km = s.chain_bk[j] != 0;
    p.bk[j] = km ? 1 : 0;
    const uint8_t* vpos = km ? rows[j] : cols[j];  // positions of the contiguous bits 0..2
    int vslot[3];
    bool used[6] = {false, false, false, false, false, false};
    for (int b = 0; b < 3; ++b) {
      vslot[b] = index6(cols[j - 1], vpos[b]);
      QSVB_REQUIRE(vslot[b] < 6, "chain pass: an operand's contiguous bits must be columns of the previous matrix");
      used[vslot[b]] = true;
    }
    int free_slots[3], nf = 0;
    for (int i = 0; i < 6; ++i)
      if (!used[i]) free_slots[nf++] = i;
    for (uint32_t e = 0; e < 8; ++e) {
      uint32_t c = 0;
      for (int b = 0; b < 3; ++b) c |= ((e >> b) & 1u) << vslot[b];
      p.ce[j][e] = uint8_t(c);
    }
    for (uint32_t m = 0; m < 4; ++m) p.cm[j][m] = uint8_t(((m & 1u) << free_slots[1]) | ((m >> 1) << free_slots[2]));
    for (uint32_t w = 0; w < 2; ++w) p.cw[j][w] = uint8_t(w << free_slots[0]);
    auto off_of = [&](uint32_t r, uint32_t c) {
      const uint32_t d = d_of(j, pos_of(j - 1, r & 63u, c));
      return b_off(km, (r >> 6) * 64u + (d >> 6), d & 63u);
    };
    for (uint32_t r = 0; r < 128; ++r) p.crow[j][r] = uint16_t(off_of(r, 0));
    for (uint32_t w = 0; w < 2; ++w)
      for (uint32_t m = 0; m < 4; ++m) p.cchunk[j][w][m] = uint16_t(off_of(0, uint32_t(p.cw[j][w]) | p.cm[j][m]));
  }
  // last matrix -> output staging at the permuted position, swizzled
  p.evec = s.chain_evec ? 1u : 0u;
  if (p.evec)
    QSVB_REQUIRE(s.chain_perm[cols[nm - 1][0]] == 0 && s.chain_perm[cols[nm - 1][1]] == 1,
                 "chain pass: vector epilogue needs the last matrix's columns 0, 1 on output bits 0, 1");
  uint32_t lane_pos[5];
  for (int b = 0; b < 5; ++b)
    lane_pos[b] = uint32_t(__builtin_ctz(permute12(1u << rows[nm - 1][b], s.chain_perm)));
  staging_swizzle(lane_pos, p.evec != 0, p.sig_lo, p.sig_hi);
  auto sig = [&](uint32_t t) { return uint32_t(p.sig_lo[t & 63u]) ^ p.sig_hi[t >> 6]; };
  for (uint32_t r = 0; r < 128; ++r)
    p.frow[r] =
        uint16_t((r >> 6) * uint32_t(kTileAmps) * 4u + 4u * sig(permute12(pos_of(nm - 1, r & 63u, 0), s.chain_perm)));
  for (uint32_t c = 0; c < 64; ++c) p.fcol[c] = uint16_t(4u * sig(permute12(pos_of(nm - 1, 0, c), s.chain_perm)));
  check_chain_params(p, nm);
  return bmode;
}

}  // namespace

// Operand layouts and orders of a pass (the planner has fixed its rows, columns and permutation):
//  * the last matrix's columns 0, 1 are the positions the permutation sends to output bits 0, 1
//    when both are its columns (vector epilogue; for a single matrix whose B is MN-major only if
//    those are state bits 0, 1 themselves);
//  * each later matrix j takes the B layout (MN- or K-major) whose contiguous bits can be three
//    columns of matrix j - 1 (columns of both, or new rows of j: one set has at least three);
//  * the three row bits of matrix j - 1 that select a converter lane within a 16-byte store phase
//    go where they spread those stores over distinct bank groups;
//  * matrix j's entries are permuted to its new row order (the column order is the kernel's own).
void tc_chain_prepare(Sweep& s) {
  QSVB_REQUIRE(s.chain_nmat >= 1 && s.chain_nmat <= uint32_t(kChainMaxMats), "chain pass: 1..3 matrices");
  const uint32_t nm = s.chain_nmat, L = nm - 1;
  for (uint32_t j = 0; j < nm; ++j)
    QSVB_REQUIRE(s.chain_mats[j].size() == 64 * 64, "chain pass: matrices are 64 x 64");
  uint8_t at_out[12];
  for (int t = 0; t < 12; ++t) at_out[s.chain_perm[t]] = uint8_t(t);
  const uint8_t q0 = at_out[0], q1 = at_out[1];
  bool evec = !contains6(s.chain_rows[L], q0) && !contains6(s.chain_rows[L], q1);
  const uint32_t bmode0 = first_bmode(s.chain_rows[0]);
  if (evec && L == 0 && bmode0 == 0 && !(q0 == 0 && q1 == 1)) evec = false;
  // first matrix: rows ascending; columns ascending, or [q0, q1, rest] for a vector epilogue
  auto put_first = [](uint8_t (&a)[6], uint8_t x, uint8_t y) {
    std::vector<uint8_t> rest;
    for (int i = 0; i < 6; ++i)
      if (a[i] != x && a[i] != y) rest.push_back(a[i]);
    std::sort(rest.begin(), rest.end());
    a[0] = x;
    a[1] = y;
    for (int i = 0; i < 4; ++i) a[2 + i] = rest[size_t(i)];
  };
  QSVB_REQUIRE(std::is_sorted(s.chain_rows[0], s.chain_rows[0] + 6), "chain pass: the first matrix's rows must ascend");
  std::sort(s.chain_cols[0], s.chain_cols[0] + 6);
  if (L == 0 && evec) put_first(s.chain_cols[0], q0, q1);
  for (uint32_t j = 1; j < nm; ++j) {
    const uint8_t(&pc)[6] = s.chain_cols[j - 1];
    std::vector<uint8_t> both, newrows;  // columns of j - 1 that are columns / rows of j
    for (int i = 0; i < 6; ++i) (contains6(s.chain_rows[j], pc[i]) ? newrows : both).push_back(pc[i]);
    bool km;
    std::vector<uint8_t> v;
    const bool fix01 = j == L && evec;
    if (fix01 && newrows.size() >= 3) {
      km = true;
      v.assign(newrows.begin(), newrows.begin() + 3);
    } else if (fix01 && both.size() >= 3 && std::count(both.begin(), both.end(), q0) &&
               std::count(both.begin(), both.end(), q1)) {
      km = false;
      v = {q0, q1};
      for (uint8_t x : both)
        if (x != q0 && x != q1 && v.size() < 3) v.push_back(x);
    } else {
      if (fix01) evec = false;
      km = both.size() < 3;
      const std::vector<uint8_t>& src = km ? newrows : both;
      v.assign(src.begin(), src.begin() + 3);
    }
    // slot assignment: contiguous bits first, then the lane bits of matrix j - 1 (its rows 0..2) on
    // the bits that pick the 16-byte bank group (K-major: row slots 3..5 and column slots 0..2;
    // MN-major: column slots 3..5 and row slots 0..2), then the rest in ascending position
    int rslot[12], cslot[12];
    for (int t = 0; t < 12; ++t) rslot[t] = cslot[t] = -1;
    bool rtaken[6] = {false}, ctaken[6] = {false};
    auto place = [&](bool is_row, uint8_t pos, int slot) {
      if (is_row) {
        rslot[pos] = slot;
        rtaken[slot] = true;
      } else {
        cslot[pos] = slot;
        ctaken[slot] = true;
      }
    };
    for (int b = 0; b < 3; ++b) place(km, v[size_t(b)], b);
    if (j == L && evec && km) {  // the last matrix's columns 0, 1 for the vector epilogue
      place(false, q0, 0);
      place(false, q1, 1);
    }
    for (int b = 0; b < 3; ++b) {
      const uint8_t pos = s.chain_rows[j - 1][b];
      const bool is_row = contains6(s.chain_rows[j], pos);
      if ((is_row ? rslot[pos] : cslot[pos]) >= 0) continue;
      // the bank-group bits for this lane bit: index b, else any free one of the three
      const int base = is_row ? (km ? 3 : 0) : (km ? 0 : 3);
      bool* taken = is_row ? rtaken : ctaken;
      int slot = -1;
      for (int k = 0; k < 3 && slot < 0; ++k) {
        const int cand = base + (b + k) % 3;
        if (!taken[cand]) slot = cand;
      }
      if (slot >= 0) place(is_row, pos, slot);
    }
    uint8_t nr[6], nc[6];
    {
      std::vector<uint8_t> rest_r, rest_c;
      for (int i = 0; i < 6; ++i) {
        if (rslot[s.chain_rows[j][i]] < 0) rest_r.push_back(s.chain_rows[j][i]);
        if (cslot[s.chain_cols[j][i]] < 0) rest_c.push_back(s.chain_cols[j][i]);
      }
      std::sort(rest_r.begin(), rest_r.end());
      std::sort(rest_c.begin(), rest_c.end());
      size_t kr = 0, kc = 0;
      for (int i = 0; i < 6; ++i) {
        if (!rtaken[i]) rslot[rest_r[kr++]] = i;
        if (!ctaken[i]) cslot[rest_c[kc++]] = i;
      }
      for (int i = 0; i < 6; ++i) {
        nr[rslot[s.chain_rows[j][i]]] = s.chain_rows[j][i];
        nc[cslot[s.chain_cols[j][i]]] = s.chain_cols[j][i];
      }
    }
    // the matrix in the new row order: index bit i now means tile position nr[i]
    int from[6];
    for (int i = 0; i < 6; ++i) from[i] = index6(s.chain_rows[j], nr[i]);
    const std::vector<cd>& m = s.chain_mats[j];
    std::vector<cd> m2(64 * 64);
    for (uint32_t r = 0; r < 64; ++r)
      for (uint32_t c = 0; c < 64; ++c) {
        uint32_t ro = 0, co = 0;
        for (int i = 0; i < 6; ++i) {
          ro |= ((r >> i) & 1u) << from[i];
          co |= ((c >> i) & 1u) << from[i];
        }
        m2[size_t(r) * 64 + c] = m[size_t(ro) * 64 + co];
      }
    s.chain_mats[j] = std::move(m2);
    std::copy(nr, nr + 6, s.chain_rows[j]);
    std::copy(nc, nc + 6, s.chain_cols[j]);
    s.chain_bk[j] = km ? 1 : 0;
  }
  s.chain_evec = evec ? 1 : 0;
}

size_t tc_chain_matrix_bytes(const Sweep& s) { return size_t(s.chain_nmat) * 2 * 128 * 128 * 2; }

// Per matrix: A = [[Ur, -Ui], [Ui, Ur]] (128 x 128), split into bf16 hi/lo, in the tensor-memory
// image order of tc_pack_matrix (hi then lo, each 128 rows x 64 words of bf16 pairs).
void tc_chain_pack(const Sweep& s, void* dst) {
  for (uint32_t j = 0; j < s.chain_nmat; ++j) {
    Sweep one;
    one.kind = SK_DENSE_TC;
    one.m = 6;
    one.mat = s.chain_mats[j];
    tc_pack_matrix(one, static_cast<char*>(dst) + size_t(j) * 2 * 128 * 128 * 2);
  }
}

void tc_chain_check(const Sweep& s, uint32_t n) {
  ChainParams p;
  TileLayout lay;
  (void)build_chain_params(s, n, nullptr, nullptr, p, lay);
}

void launch_tc_chain(const LaunchEnv& env, float* re, float* im, uint32_t n, const Sweep& s, const void* dev_mat) {
  QSVB_REQUIRE(env.err_flag != nullptr, "chain pass needs the context error flag");
  ChainParams p;
  TileLayout lay;
  const uint32_t bmode = build_chain_params(s, n, re, im, p, lay);
  const uint64_t ntiles = 1ull << (n - 12);
  // up to two matrices: four accumulators (tiles in flight); three matrices leave tensor memory for two
  using Kern = decltype(&k_tc_chain<0, 2>);
  static const Kern kerns[2][4] = {{k_tc_chain<0, 2>, k_tc_chain<1, 2>, k_tc_chain<2, 2>, k_tc_chain<3, 2>},
                                   {k_tc_chain<0, 4>, k_tc_chain<1, 4>, k_tc_chain<2, 4>, k_tc_chain<3, 4>}};
  const Kern kern = kerns[s.chain_nmat <= 2 ? 1 : 0][bmode];
  QSVB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kChainSmem)));
  QSVB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                               int(cudaSharedmemCarveoutMaxShared)));
  // one persistent CTA per SM (the tensor-memory allocation of 512 columns assumes it)
  const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(env.num_sms))));
  kern<<<grid, kThreads, kChainSmem, env.stream>>>(re, im, ntiles, static_cast<const uint4*>(dev_mat), p,
                                                     env.err_flag, lay.maps[0], lay.maps[1]);
  QSVB_CK(cudaGetLastError());
}

template <class R>
void launch_permute(const LaunchEnv& env, R* re, R* im, uint32_t n, const Sweep& s) {
  QSVB_REQUIRE(n >= 12, "permutation pass: state too small");
  PermParams p;
  std::memset(&p, 0, sizeof(p));
  TileLayout lay;
  tile_layout(n, s.chain_tbits, nullptr, nullptr, lay);
  std::copy(lay.hibits, lay.hibits + 6, p.hibits);
  std::copy(lay.hioff, lay.hioff + 64, p.hioff);
  for (uint32_t i = 0; i < 64; ++i) {
    p.plo[i] = uint16_t(permute12(i, s.chain_perm));
    p.phi[i] = uint16_t(permute12(i << 6, s.chain_perm));
  }
  const uint64_t ntiles = 1ull << (n - 12);
  const size_t smem = 2 * sizeof(R) * kTileAmps;
  QSVB_CK(cudaFuncSetAttribute(k_permute_tiles<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  int occ = 0;
  QSVB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_permute_tiles<R>, kPermThreads, smem));
  QSVB_REQUIRE(occ >= 1, "permutation kernel does not fit on an SM");
  const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(env.num_sms) * occ)));
  k_permute_tiles<R><<<grid, kPermThreads, smem, env.stream>>>(re, im, ntiles, p);
  QSVB_CK(cudaGetLastError());
}
template void launch_permute<float>(const LaunchEnv&, float*, float*, uint32_t, const Sweep&);
template void launch_permute<double>(const LaunchEnv&, double*, double*, uint32_t, const Sweep&);

}  // namespace qsvb
