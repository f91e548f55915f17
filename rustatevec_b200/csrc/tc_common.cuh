// Shared pieces of the tcgen05 kernels (tc_dense.cu, tc_chain.cu): inline-PTX wrappers for
// tensor memory, MMA issue, mbarriers and bulk/tensor copies (no multicast anywhere), the
// 128-byte-swizzled operand layouts, the output staging swizzle, host-side bf16 rounding, and the
// address layout of a 4096-amplitude tile.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

namespace qsvb {
namespace tc {

constexpr long long kWaitBudget = 1ll << 31;  // clock64 cycles (~1 s) for every bounded mbarrier wait

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

// A from tensor memory (M rows in lanes, K packed two bf16 per 32-bit column), B from shared.
__device__ __forceinline__ void mma_bf16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t idesc,
                                            uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc));
}

// One lane of a converged warp (the lowest), as a 0/1 flag. An MMA role keeps the whole warp on
// uniform control flow and lets this lane issue: the operands then stay warp-uniform, and one
// tcgen05.mma issues about every 37 cycles (N = 64) instead of about every 80 from a branch taken by
// lane 0 alone.
__device__ __forceinline__ uint32_t elect_one() {
  uint32_t r;
  asm volatile("{\n\t.reg .pred e;\n\telect.sync _|e, 0xffffffff;\n\tselp.u32 %0, 1, 0, e;\n\t}\n" : "=r"(r));
  return r;
}

// mma_bf16_ts / mma_commit issued by the lane whose `leader` flag is set (the rest of the warp
// executes the same instruction stream with the predicate off).
__device__ __forceinline__ void mma_bf16_ts_by(uint32_t leader, uint32_t d_tmem, uint32_t a_tmem, uint64_t b,
                                               uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p, e;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "setp.ne.b32 e, %5, 0;\n\t"
      "@e tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc), "r"(leader));
}

__device__ __forceinline__ void mma_commit_by(uint32_t leader, uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .pred e;\n\tsetp.ne.b32 e, %1, 0;\n\t"
      "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}\n" ::"r"(smem_u32(bar)),
      "r"(leader)
      : "memory");
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

// Arrive on behalf of `count` of the barrier's expected arrivals.
__device__ __forceinline__ void mbar_arrive_cnt(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// A waiting thread is suspended in hardware until the phase completes (or the hint, 1 ms, runs out),
// so waiting roles do not spin on the barrier and take issue slots from the working warps.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(1000000u)
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

// Same, adding the cycles spent waiting to `acc` (stall profiling).
__device__ __forceinline__ bool mbar_wait_t(uint64_t* bar, uint32_t parity, long long& acc) {
  const long long t0 = clock64();
  const bool ok = mbar_wait(bar, parity);
  acc += clock64() - t0;
  return ok;
}

// 32 lanes x 32 fp32 columns, and the wait for it, in one statement: the registers are defined only
// once the load has completed (a separate tcgen05.wait::ld does not stop the compiler from
// scheduling register-only uses of the loaded values before the wait).
__device__ __forceinline__ void tmem_ld32_wait(uint32_t addr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(addr)
      : "memory");
}
// 32 lanes x 64 fp32 columns (two loads of 32) and the wait, in one statement.
__device__ __forceinline__ void tmem_ld64_wait(uint32_t addr, uint32_t (&r)[64]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%64];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%65];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
      : "r"(addr), "r"(addr + 32u)
      : "memory");
}

// 32 lanes x 64 32-bit columns from registers (one lane per thread of the warp).
__device__ __forceinline__ void tmem_st64(uint32_t addr, const uint32_t (&r)[64]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x64.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,"
      "%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63,%64};\n" ::"r"(addr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
      "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]),
      "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]),
      "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31]), "r"(r[32]), "r"(r[33]), "r"(r[34]), "r"(r[35]), "r"(r[36]),
      "r"(r[37]), "r"(r[38]), "r"(r[39]), "r"(r[40]), "r"(r[41]), "r"(r[42]), "r"(r[43]), "r"(r[44]), "r"(r[45]),
      "r"(r[46]), "r"(r[47]), "r"(r[48]), "r"(r[49]), "r"(r[50]), "r"(r[51]), "r"(r[52]), "r"(r[53]), "r"(r[54]),
      "r"(r[55]), "r"(r[56]), "r"(r[57]), "r"(r[58]), "r"(r[59]), "r"(r[60]), "r"(r[61]), "r"(r[62]), "r"(r[63])
      : "memory");
}

__device__ __forceinline__ void named_sync(uint32_t id, uint32_t nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
// Named barrier that also returns whether `v` holds for every participating thread.
__device__ __forceinline__ bool named_all(uint32_t id, uint32_t nthreads, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"(uint32_t(v)), "r"(id), "r"(nthreads)
      : "memory");
  return r != 0;
}

// Shared-memory accesses by 32-bit shared address (explicit state space).
__device__ __forceinline__ float4 lds128f(uint32_t a) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a)
               : "memory");
  return v;
}
__device__ __forceinline__ void sts64(uint32_t a, uint32_t x, uint32_t y) {
  asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(a), "r"(x), "r"(y) : "memory");
}
__device__ __forceinline__ void sts32(uint32_t a, uint32_t x) {
  asm volatile("st.shared.b32 [%0], %1;" ::"r"(a), "r"(x) : "memory");
}
__device__ __forceinline__ void sts128f(uint32_t a, float4 v) {
  asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w) : "memory");
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
__host__ __device__ __forceinline__ uint32_t kmaj_off(uint32_t row, uint32_t kk, uint32_t rows) {
  return (kk >> 6) * (rows * 128u) + (row >> 3) * 1024u + (row & 7u) * 128u +
         ((((kk & 63u) >> 3) ^ (row & 7u)) << 4) + (kk & 7u) * 2u;
}
// Byte offset in an MN-major, 128-byte-swizzled operand of 64 columns (one atom wide).
__host__ __device__ __forceinline__ uint32_t mnmaj_off(uint32_t kk, uint32_t col) {
  return (kk >> 3) * 1024u + (kk & 7u) * 128u + ((((col >> 3) ^ (kk & 7u))) << 4) + (col & 7u) * 2u;
}
// Output staging (fp32, address order) with a 16-byte XOR swizzle against bank conflicts.
// XOR-linear: stage_idx(a ^ b) = stage_idx(a) ^ stage_idx(b), so an index assembled from disjoint
// row and column bits can be swizzled part by part.
__host__ __device__ __forceinline__ uint32_t stage_idx(uint32_t t) { return t ^ (((t >> 7) & 7u) << 2); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// One tiled tensor-map copy global -> this CTA's shared memory (no multicast), rank 1..5.
__device__ __forceinline__ void tma_tensor_g2s(void* dst, const CUtensorMap* map, const int (&c)[5], uint32_t rank,
                                               uint64_t* bar) {
  const uint64_t m = reinterpret_cast<uint64_t>(map);
  const uint32_t d = smem_u32(dst), b = smem_u32(bar);
  switch (rank) {
    case 1:
      asm volatile("cp.async.bulk.tensor.1d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2}], [%3];"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(b) : "memory");
      break;
    case 2:
      asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(b) : "memory");
      break;
    case 3:
      asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(b) : "memory");
      break;
    case 4:
      asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(b) : "memory");
      break;
    default:
      asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(b) : "memory");
      break;
  }
}

// A whole tile in address order by tiled tensor-map copies (no multicast): one per value of the
// `nouter` tile bits folded into the last dimension's coordinate (bit positions obit), each filling
// the next 4096 >> nouter amplitudes of the slot. `base` is the tile's first state index.
__device__ __forceinline__ void tma_tile_g2s(float* dre, float* dim, const CUtensorMap* mre, const CUtensorMap* mim,
                                             uint64_t base, uint32_t rank, const uint32_t (&start)[5],
                                             const uint32_t (&len)[5], uint32_t nouter, const uint32_t (&obit)[3],
                                             uint64_t* bar) {
  int c[5];
#pragma unroll
  for (uint32_t d = 0; d < 5; ++d) c[d] = d < rank ? int((base >> start[d]) & ((1ull << len[d]) - 1ull)) : 0;
  const uint32_t chunk = 4096u >> nouter;
  for (uint32_t o = 0; o < (1u << nouter); ++o) {
    int cc[5] = {c[0], c[1], c[2], c[3], c[4]};
    for (uint32_t k = 0; k < nouter; ++k) cc[rank - 1] |= int(((o >> k) & 1u) << obit[k]);
    tma_tensor_g2s(dre + o * chunk, mre, cc, rank, bar);
    tma_tensor_g2s(dim + o * chunk, mim, cc, rank, bar);
  }
}

// One bulk copy global -> this CTA's shared memory, completing on `bar` (no multicast).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// ---------------------------------------------------------------- host-side bf16 rounding
inline uint16_t bf16_bits_rn(float x) {  // round-to-nearest-even, finite inputs
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return uint16_t(u >> 16);
}
inline float bf16_to_float(uint16_t h) {
  const uint32_t u = uint32_t(h) << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}


}  // namespace tc

constexpr int kTileBitsAll = 12;  // a tensor-core tile is 2^12 amplitudes

// Address layout of a 4096-amplitude tile whose bits are `tbits` (ascending; bits 0..5 always
// among them): the offsets of the high six tile bits, the length of the contiguous low run, and,
// when that run is short, a tensor map per component whose box is exactly the tile.
struct TileLayout {
  uint32_t hibits[6];
  uint64_t hioff[64];     // address offset of each value of the high six tile bits
  uint32_t runbits;       // log2 of the contiguous run length (>= 6)
  uint32_t tm_rank;       // > 0: tiled tensor-map copies fetch the tile (2^tm_outer per component)
  uint32_t tm_start[5], tm_len[5];
  uint32_t tm_box[5];     // log2 of each dimension's box extent (its run of tile bits)
  uint32_t tm_outer;      // tile bits folded into the last dimension's coordinate (0..3)
  uint32_t tm_obit[3];    // their bit positions in that coordinate
  CUtensorMap maps[2];
};
void tile_layout(uint32_t n, const uint32_t (&tbits)[12], float* re, float* im, TileLayout& out);

}  // namespace qsvb
