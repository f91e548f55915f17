// Batched execution of many small independent circuits in one persistent kernel.
//
// Host plan. Each circuit is split into passes over HBM: a pass owns a set S of at most L local
// qubits (always including state bits 0-4, so global accesses are runs of >= 32 contiguous
// amplitudes) and takes the gates that act inside S and commute past every gate left for later
// passes (gates on disjoint qubits). A circuit with n <= L is a single pass whose whole state lives
// in one thread block's shared memory: |0..0> is built there and only the FP64 probabilities and
// <Z_0> leave the SM. Larger circuits keep their state in HBM; a pass is 2^(n-|S|) disjoint tiles of
// 2^|S| amplitudes (the non-local bits fixed), each loaded into shared memory, updated and written
// back (the first pass starts from |0..0> without reading, the last writes probabilities instead of
// the state).
//
// Inside a pass the gates are split the same way once more into register phases: a phase owns RB
// local positions (5 for complex64, 4 for complex128); a thread holds a group of 2^RB amplitudes
// that share the other local bits in registers, applies all of the phase's gates there, and writes
// them back (256 threads, up to 512 groups per phase). Shared memory is touched once per phase
// instead of once per gate. The shared-memory index is XOR-swizzled (a linear map on the index
// bits) and each phase picks which non-register positions become warp lanes so that a warp's 32
// accesses fall in distinct banks.
//
// Work items are (pass, tile) pairs in one queue ordered level by level (pass 0 of every circuit,
// then pass 1, ...), costliest circuits first within a level, so every item's dependencies are
// earlier in the queue and were taken by a running block. A persistent grid takes items with an
// atomic counter; a tile of pass p spins, with a clock64 budget, until all tiles of pass p-1 of its
// circuit are done. A spin that runs out sets the context's error flag and later waits give up at
// once (the host reports QSVB_E_TIMEOUT). <Z_0> partial sums go to one slot per last-pass tile and
// are summed per circuit in a fixed order afterwards, so results are deterministic. The per-run
// device work (counter resets, the persistent kernel, the <Z_0> sums) is one CUDA graph per batch.

#include <cuda/atomic>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <future>
#include <memory>
#include <mutex>
#include <numeric>
#include <type_traits>
#include <string>
#include <thread>
#include <vector>

#include "qsvb_internal.h"

namespace qsvb {
namespace {

constexpr int kMaxLocal = 14;
constexpr int kMaxHi = 512;                   // 2^(kMaxLocal - 5): entries of the address / swizzle tables
constexpr long long kSpinBudget = 1ll << 32;  // default dependency-wait budget, clock64 cycles (about 2 s)
constexpr uint32_t kStageBytes = 32768;       // shared memory for one pass's program
// The same for tile sweeps: small enough for five blocks per SM (larger programs are read from
// global memory through L1).
constexpr uint32_t kTileStageBytes = 8192;
constexpr int kTileHi = 128;  // address / swizzle table entries of tile sweeps (<= 12 local bits)

// OP_D1T: a diagonal on one register bit whose two entries depend on one bit of the tile index
// (a 2-qubit diagonal with one qubit outside the tile); OP_DT: a phase that depends only on tile
// bits (a diagonal whose qubits are all outside the tile), applied to every amplitude.
// OP_D1P / OP_DTP: the same as OP_D1 / OP_DT with coefficients computed once per tile from a
// phase sum over tile bits (tile sweeps merge runs of diagonal gates into them).
enum BatchOp : uint32_t {
  OP_PHASE = 0, OP_1Q = 1, OP_D1 = 2, OP_CX = 3, OP_2Q = 4, OP_D2 = 5, OP_D1T = 6, OP_DT = 7, OP_D1P = 8, OP_DTP = 9,
  OP_DTAB = 10,  // the product of a phase's diagonal gates: one factor per register slot
  OP_1QR = 11,   // a real 1-qubit gate [[a, b], [c, d]] (RY, H, X): half the work of a general one
  OP_1QX = 12,   // [[a, i b], [i c, d]] with a..d real (RX, Y): half the work as well
  OP_D1G = 13    // a diagonal on one register bit whose entries depend on bits of the group index
};
constexpr uint32_t kTphSlots = 32;  // per-tile phase operations per pass (tile sweeps)
constexpr uint32_t kTphSlotR = 12;  // reals per slot (the OP_D1 coefficient block of either precision)

struct Instr {
  uint32_t op;
  uint32_t a, b;  // register bits (1Q/D1/D1T: a; CX: a = control, b = target; 2Q/D2: a < b, matrix bit 0 <->
                  // a); D1T: b = tile bit; DT: b = tile bit of entry bit 0 | (tile bit of entry bit 1
                  // << 8) | (number of tile bits << 16)
  uint32_t coef;  // complex index into the coefficient array (OP_PHASE: phase index)
};

struct PhaseDev {
  uint32_t rphys[5];  // swizzled shared-memory offset of each register bit's unit vector
  uint32_t r, nt;     // register bits used, group bits (2^nt groups of 2^r amplitudes)
  uint32_t ninstr;    // gate instructions that follow the phase instruction
  // swizzled shared-memory offset of a group's first amplitude, split by the group index's low 5
  // bits (the warp lanes) and the bits above: offset(g) = lo[g & 31] ^ hi[g >> 5]
  uint16_t lo[32], hi[32];
};

struct PassDev {
  uint32_t circuit, nlocal, first, last;
  uint32_t prog_off, prog_len, ntiles, prev;  // prev: previous pass of the same circuit (or ~0u)
  uint32_t nnon;
  uint8_t nonlocal[32];  // non-local state bits, ascending
  uint8_t local[16];     // local position -> state bit, ascending
  uint64_t state_off;    // amplitude offset of the circuit's state
  uint64_t prob_off;     // offset of the circuit's probabilities
  uint64_t zslot;        // first <Z_0> partial slot (last pass)
  uint32_t phase_off, nphase, coef_off, ncoef;  // the pass's phases and coefficients (complex units)
  uint32_t staged;       // program fits the shared-memory staging area
  uint32_t tph_n, tph_off;  // per-tile phase sums: count and byte offset from this record
};

struct Item {
  uint32_t pass;
  uint32_t tile;
};

// Swizzle: shared-memory slot = x ^ (XOR over set bits p >= W of x of col(p)), a linear bijection
// that only changes the low W bits (W = 5 for 4-byte words, 4 for 8-byte words: the bits that pick
// the bank for a warp, or for each half-warp with 8-byte words).
__host__ __device__ inline uint32_t swz_col(int p, int W) {
  if (p < W) return 0u;
  if (p < 2 * W) return 1u << (p - W);
  return (1u << (W - 1)) | (1u << ((p - 2 * W) % (W - 1)));
}

// One amplitude component global -> shared without a register round trip (many in flight).
template <class R>
__device__ __forceinline__ void cp_async_elem(R* dst, const R* src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  if constexpr (sizeof(R) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}

// 16-byte vectors of amplitude components (4 floats / 2 doubles) for the tile fill and write-back.
template <class R> struct Vec16;
template <> struct Vec16<float> {
  using T = float4;
  static constexpr int N = 4;
  __device__ static float get(const float4& v, int e) { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; }
  __device__ static void set(float4& v, int e, float x) {
    if (e == 0) v.x = x; else if (e == 1) v.y = x; else if (e == 2) v.z = x; else v.w = x;
  }
};
template <> struct Vec16<double> {
  using T = double2;
  static constexpr int N = 2;
  __device__ static double get(const double2& v, int e) { return e == 0 ? v.x : v.y; }
  __device__ static void set(double2& v, int e, double x) {
    if (e == 0) v.x = x; else v.y = x;
  }
};

template <class R>
__device__ __forceinline__ void cmac(R& yr, R& yi, R ar, R ai, R xr, R xi) {
  yr = fma(ar, xr, yr);
  yr = fma(-ai, xi, yr);
  yi = fma(ar, xi, yi);
  yi = fma(ai, xr, yi);
}

// ---- register storage of one group: complex64 keeps amplitude pairs (s, s^1) in float2 registers
// so a gate on any register bit but 0 runs on Blackwell's paired FP32 FMA (two amplitudes per
// instruction); complex128 keeps one amplitude per register.
template <class R, int RB> struct Regs;
template <int RB> struct Regs<float, RB> {
  float2 r[(1 << RB) / 2], i[(1 << RB) / 2];
  __device__ __forceinline__ float& re(int s) { return (s & 1) ? r[s >> 1].y : r[s >> 1].x; }
  __device__ __forceinline__ float& im(int s) { return (s & 1) ? i[s >> 1].y : i[s >> 1].x; }
};
template <int RB> struct Regs<double, RB> {
  double r[1 << RB], i[1 << RB];
  __device__ __forceinline__ double& re(int s) { return r[s]; }
  __device__ __forceinline__ double& im(int s) { return i[s]; }
};

// ---- gates on register bits (compile-time bit positions, so the amplitudes stay in registers)
template <int J, class R, int RB>
__device__ __forceinline__ void g1q(Regs<R, RB>& v, const R* __restrict__ c) {
  if constexpr (J < RB) {
    if constexpr (std::is_same<R, float>::value) {
      // complex64 coefficients come pre-broadcast as float2 pairs: for each of a, b, c, d (the 2x2
      // in row-major order) the pairs (re, re), (im, im), (-im, -im)
      const float2* cc = reinterpret_cast<const float2*>(c);
      if constexpr (J >= 1) {
        // two amplitudes per instruction; same operation order as the scalar path below
        constexpr int HJ = 1 << (J - 1);
        const float2 A0 = cc[0], A1 = cc[1], NA1 = cc[2], B0 = cc[3], B1 = cc[4], NB1 = cc[5];
        const float2 C0 = cc[6], C1 = cc[7], NC1 = cc[8], D0 = cc[9], D1 = cc[10], ND1 = cc[11];
#pragma unroll
        for (int h = 0; h < (1 << RB) / 2; ++h) {
          if (h & HJ) continue;
          const int t = h | HJ;
          const float2 xr0 = v.r[h], xi0 = v.i[h], xr1 = v.r[t], xi1 = v.i[t];
          float2 yr0 = __fmul2_rn(A0, xr0), yi0 = __fmul2_rn(A0, xi0);
          float2 yr1 = __fmul2_rn(C0, xr0), yi1 = __fmul2_rn(C0, xi0);
          yr0 = __ffma2_rn(NA1, xi0, yr0);
          yi0 = __ffma2_rn(A1, xr0, yi0);
          yr1 = __ffma2_rn(NC1, xi0, yr1);
          yi1 = __ffma2_rn(C1, xr0, yi1);
          yr0 = __ffma2_rn(B0, xr1, yr0);
          yi0 = __ffma2_rn(B0, xi1, yi0);
          yr1 = __ffma2_rn(D0, xr1, yr1);
          yi1 = __ffma2_rn(D0, xi1, yi1);
          yr0 = __ffma2_rn(NB1, xi1, yr0);
          yi0 = __ffma2_rn(B1, xr1, yi0);
          yr1 = __ffma2_rn(ND1, xi1, yr1);
          yi1 = __ffma2_rn(D1, xr1, yi1);
          v.r[h] = yr0;
          v.i[h] = yi0;
          v.r[t] = yr1;
          v.i[t] = yi1;
        }
      } else {
        const float a0 = cc[0].x, a1 = cc[1].x, b0 = cc[3].x, b1 = cc[4].x;
        const float c0 = cc[6].x, c1 = cc[7].x, d0 = cc[9].x, d1 = cc[10].x;
#pragma unroll
        for (int h = 0; h < (1 << RB) / 2; ++h) {
          const float xr0 = v.r[h].x, xi0 = v.i[h].x, xr1 = v.r[h].y, xi1 = v.i[h].y;
          float yr0 = a0 * xr0, yi0 = a0 * xi0, yr1 = c0 * xr0, yi1 = c0 * xi0;
          yr0 = fmaf(-a1, xi0, yr0);
          yi0 = fmaf(a1, xr0, yi0);
          yr1 = fmaf(-c1, xi0, yr1);
          yi1 = fmaf(c1, xr0, yi1);
          yr0 = fmaf(b0, xr1, yr0);
          yi0 = fmaf(b0, xi1, yi0);
          yr1 = fmaf(d0, xr1, yr1);
          yi1 = fmaf(d0, xi1, yi1);
          yr0 = fmaf(-b1, xi1, yr0);
          yi0 = fmaf(b1, xr1, yi0);
          yr1 = fmaf(-d1, xi1, yr1);
          yi1 = fmaf(d1, xr1, yi1);
          v.r[h] = make_float2(yr0, yr1);
          v.i[h] = make_float2(yi0, yi1);
        }
      }
    } else {
      const R a0 = c[0], a1 = c[1], b0 = c[2], b1 = c[3], c0 = c[4], c1 = c[5], d0 = c[6], d1 = c[7];
#pragma unroll
      for (int s = 0; s < (1 << RB); ++s) {
        if (s & (1 << J)) continue;
        const int t = s | (1 << J);
        const R xr0 = v.re(s), xi0 = v.im(s), xr1 = v.re(t), xi1 = v.im(t);
        R yr0 = a0 * xr0, yi0 = a0 * xi0, yr1 = c0 * xr0, yi1 = c0 * xi0;
        yr0 = fma(-a1, xi0, yr0);
        yi0 = fma(a1, xr0, yi0);
        yr1 = fma(-c1, xi0, yr1);
        yi1 = fma(c1, xr0, yi1);
        yr0 = fma(b0, xr1, yr0);
        yi0 = fma(b0, xi1, yi0);
        yr1 = fma(d0, xr1, yr1);
        yi1 = fma(d0, xi1, yi1);
        yr0 = fma(-b1, xi1, yr0);
        yi0 = fma(b1, xr1, yi0);
        yr1 = fma(-d1, xi1, yr1);
        yi1 = fma(d1, xr1, yi1);
        v.re(s) = yr0;
        v.im(s) = yi0;
        v.re(t) = yr1;
        v.im(t) = yi1;
      }
    }
  }
}

template <int J, class R, int RB>
__device__ __forceinline__ void gd1(Regs<R, RB>& v, const R* __restrict__ c) {
  if constexpr (J < RB) {
    if constexpr (std::is_same<R, float>::value) {
      // pre-broadcast pairs (re, im, -im) for the 0 side and the 1 side of bit J; for J == 0 the
      // pair (s, s^1) straddles bit J, so both sets hold (value at s, value at s^1)
      const float2* cc = reinterpret_cast<const float2*>(c);
      const float2 pr0 = cc[0], pi0 = cc[1], npi0 = cc[2], pr1 = cc[3], pi1 = cc[4], npi1 = cc[5];
#pragma unroll
      for (int h = 0; h < (1 << RB) / 2; ++h) {
        const bool one = J >= 1 && (h & (1 << (J >= 1 ? J - 1 : 0)));
        const float2 pr = one ? pr1 : pr0, pi = one ? pi1 : pi0, npi = one ? npi1 : npi0;
        const float2 xr = v.r[h], xi = v.i[h];
        v.r[h] = __ffma2_rn(pr, xr, __fmul2_rn(npi, xi));
        v.i[h] = __ffma2_rn(pr, xi, __fmul2_rn(pi, xr));
      }
    } else {
      const R p0r = c[0], p0i = c[1], p1r = c[2], p1i = c[3];
#pragma unroll
      for (int s = 0; s < (1 << RB); ++s) {
        const R pr = (s & (1 << J)) ? p1r : p0r, pi = (s & (1 << J)) ? p1i : p0i;
        const R xr = v.re(s), xi = v.im(s);
        v.re(s) = fma(pr, xr, -pi * xi);
        v.im(s) = fma(pr, xi, pi * xr);
      }
    }
  }
}

// Diagonal on register bit J whose entries depend on bits of this thread's group index gidx (local
// qubits outside the phase's registers, constant per group): for each set bit k of mask, in
// ascending order, c holds the four entries of one 2-qubit diagonal (index: register bit | group
// bit k << 1, complex pairs). The thread multiplies the entries its group bits select, then applies
// the resulting diag(f0, f1).
template <int J, class R, int RB>
__device__ __forceinline__ void gd1g(Regs<R, RB>& v, const R* __restrict__ c, uint32_t mask, uint32_t gidx) {
  if constexpr (J < RB) {
    R f0r = 1, f0i = 0, f1r = 1, f1i = 0;
    for (uint32_t mm = mask; mm; mm &= mm - 1u, c += 8) {
      const R* d = c + 4 * ((gidx >> (__ffs(mm) - 1)) & 1u);
      const R a0r = d[0], a0i = d[1], a1r = d[2], a1i = d[3];
      const R t0 = f0r * a0r - f0i * a0i, t1 = f1r * a1r - f1i * a1i;
      f0i = f0r * a0i + f0i * a0r;
      f1i = f1r * a1i + f1i * a1r;
      f0r = t0;
      f1r = t1;
    }
    if constexpr (std::is_same<R, float>::value) {
#pragma unroll
      for (int h = 0; h < (1 << RB) / 2; ++h) {
        float2 pr, pi;
        if constexpr (J == 0) {  // the pair (2h, 2h+1) straddles bit 0
          pr = make_float2(f0r, f1r);
          pi = make_float2(f0i, f1i);
        } else {
          const bool one = (h >> (J - 1)) & 1;
          pr = one ? make_float2(f1r, f1r) : make_float2(f0r, f0r);
          pi = one ? make_float2(f1i, f1i) : make_float2(f0i, f0i);
        }
        const float2 npi = make_float2(-pi.x, -pi.y);
        const float2 xr = v.r[h], xi = v.i[h];
        v.r[h] = __ffma2_rn(pr, xr, __fmul2_rn(npi, xi));
        v.i[h] = __ffma2_rn(pr, xi, __fmul2_rn(pi, xr));
      }
    } else {
#pragma unroll
      for (int s = 0; s < (1 << RB); ++s) {
        const R pr = (s & (1 << J)) ? f1r : f0r, pi = (s & (1 << J)) ? f1i : f0i;
        const R xr = v.re(s), xi = v.im(s);
        v.re(s) = fma(pr, xr, -pi * xi);
        v.im(s) = fma(pr, xi, pi * xr);
      }
    }
  }
}

template <int J, int K, class R, int RB>
__device__ __forceinline__ void gcx(Regs<R, RB>& v) {
  if constexpr (J < RB && K < RB && J != K) {
#pragma unroll
    for (int s = 0; s < (1 << RB); ++s) {
      if (!(s & (1 << J)) || (s & (1 << K))) continue;
      const int t = s | (1 << K);
      const R tr = v.re(s), ti = v.im(s);
      v.re(s) = v.re(t);
      v.im(s) = v.im(t);
      v.re(t) = tr;
      v.im(t) = ti;
    }
  }
}

template <int J, int K, class R, int RB>
__device__ __forceinline__ void g2q(Regs<R, RB>& v, const R* __restrict__ c) {
  if constexpr (J < K && K < RB) {
#pragma unroll
    for (int s = 0; s < (1 << RB); ++s) {
      if (s & ((1 << J) | (1 << K))) continue;
      const int idx[4] = {s, s | (1 << J), s | (1 << K), s | (1 << J) | (1 << K)};
      R xr[4], xi[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        xr[q] = v.re(idx[q]);
        xi[q] = v.im(idx[q]);
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        R yr = 0, yi = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) cmac(yr, yi, c[2 * (4 * r + q)], c[2 * (4 * r + q) + 1], xr[q], xi[q]);
        v.re(idx[r]) = yr;
        v.im(idx[r]) = yi;
      }
    }
  }
}

template <int J, int K, class R, int RB>
__device__ __forceinline__ void gd2(Regs<R, RB>& v, const R* __restrict__ c) {
  if constexpr (J < K && K < RB) {
#pragma unroll
    for (int s = 0; s < (1 << RB); ++s) {
      const int d = ((s >> J) & 1) | (((s >> K) & 1) << 1);
      const R pr = c[2 * d], pi = c[2 * d + 1];
      const R xr = v.re(s), xi = v.im(s);
      v.re(s) = fma(pr, xr, -pi * xi);
      v.im(s) = fma(pr, xi, pi * xr);
    }
  }
}

// A 1-qubit gate whose entries are each real or imaginary, on register bit J: X false, the real
// matrix [[a, b], [c, d]]; X true, [[a, i b], [i c, d]]. Four real multiplies per amplitude instead
// of eight. Coefficients: complex128 (a, b), (c, d); complex64 float2 pairs broadcast on the host,
// (a, a), (b, b), (c, c), (d, d) and, for X, (-b, -b), (-c, -c) after them.
template <int J, class R, int RB, bool X>
__device__ __forceinline__ void g1qs(Regs<R, RB>& v, const R* __restrict__ c) {
  if constexpr (J < RB) {
    if constexpr (std::is_same<R, float>::value) {
      const float2* cc = reinterpret_cast<const float2*>(c);
      const float2 A = cc[0], B = cc[1], Cc = cc[2], D = cc[3];
      if constexpr (J >= 1) {
        constexpr int HJ = 1 << (J - 1);
#pragma unroll
        for (int h = 0; h < (1 << RB) / 2; ++h) {
          if (h & HJ) continue;
          const int t = h | HJ;
          const float2 xr0 = v.r[h], xi0 = v.i[h], xr1 = v.r[t], xi1 = v.i[t];
          if constexpr (X) {
            const float2 NB = cc[4], NC = cc[5];
            v.r[h] = __ffma2_rn(NB, xi1, __fmul2_rn(A, xr0));
            v.i[h] = __ffma2_rn(B, xr1, __fmul2_rn(A, xi0));
            v.r[t] = __ffma2_rn(D, xr1, __fmul2_rn(NC, xi0));
            v.i[t] = __ffma2_rn(D, xi1, __fmul2_rn(Cc, xr0));
          } else {
            v.r[h] = __ffma2_rn(B, xr1, __fmul2_rn(A, xr0));
            v.i[h] = __ffma2_rn(B, xi1, __fmul2_rn(A, xi0));
            v.r[t] = __ffma2_rn(D, xr1, __fmul2_rn(Cc, xr0));
            v.i[t] = __ffma2_rn(D, xi1, __fmul2_rn(Cc, xi0));
          }
        }
      } else {
        const float a = A.x, b = B.x, cs = Cc.x, d = D.x;
#pragma unroll
        for (int h = 0; h < (1 << RB) / 2; ++h) {
          const float xr0 = v.r[h].x, xi0 = v.i[h].x, xr1 = v.r[h].y, xi1 = v.i[h].y;
          if constexpr (X) {
            v.r[h] = make_float2(fmaf(-b, xi1, a * xr0), fmaf(d, xr1, -cs * xi0));
            v.i[h] = make_float2(fmaf(b, xr1, a * xi0), fmaf(d, xi1, cs * xr0));
          } else {
            v.r[h] = make_float2(fmaf(b, xr1, a * xr0), fmaf(d, xr1, cs * xr0));
            v.i[h] = make_float2(fmaf(b, xi1, a * xi0), fmaf(d, xi1, cs * xi0));
          }
        }
      }
    } else {
      const R a = c[0], b = c[1], cs = c[2], d = c[3];
#pragma unroll
      for (int s = 0; s < (1 << RB); ++s) {
        if (s & (1 << J)) continue;
        const int t = s | (1 << J);
        const R xr0 = v.re(s), xi0 = v.im(s), xr1 = v.re(t), xi1 = v.im(t);
        if constexpr (X) {
          v.re(s) = fma(-b, xi1, a * xr0);
          v.im(s) = fma(b, xr1, a * xi0);
          v.re(t) = fma(d, xr1, -cs * xi0);
          v.im(t) = fma(d, xi1, cs * xr0);
        } else {
          v.re(s) = fma(b, xr1, a * xr0);
          v.im(s) = fma(b, xi1, a * xi0);
          v.re(t) = fma(d, xr1, cs * xr0);
          v.im(t) = fma(d, xi1, cs * xi0);
        }
      }
    }
  }
}

// One factor per register slot (a phase's diagonal gates multiplied out on the host). complex64:
// per float2 pair h the factors of slots 2h and 2h+1 as (re), (im), (-im) pairs; complex128: one
// complex per slot.
template <class R, int RB>
__device__ __forceinline__ void gtab(Regs<R, RB>& v, const R* __restrict__ c) {
  if constexpr (std::is_same<R, float>::value) {
    const float2* cc = reinterpret_cast<const float2*>(c);
#pragma unroll
    for (int h = 0; h < (1 << RB) / 2; ++h) {
      const float2 pr = cc[3 * h], pi = cc[3 * h + 1], npi = cc[3 * h + 2];
      const float2 xr = v.r[h], xi = v.i[h];
      v.r[h] = __ffma2_rn(pr, xr, __fmul2_rn(npi, xi));
      v.i[h] = __ffma2_rn(pr, xi, __fmul2_rn(pi, xr));
    }
  } else {
#pragma unroll
    for (int s = 0; s < (1 << RB); ++s) {
      const R pr = c[2 * s], pi = c[2 * s + 1];
      const R xr = v.re(s), xi = v.im(s);
      v.re(s) = fma(pr, xr, -pi * xi);
      v.im(s) = fma(pr, xi, pi * xr);
    }
  }
}

#define QSVB_PAIR_CASES(F, ...)                       \
  case 0 * 8 + 1: F<0, 1, R, RB>(__VA_ARGS__); break; \
  case 0 * 8 + 2: F<0, 2, R, RB>(__VA_ARGS__); break; \
  case 0 * 8 + 3: F<0, 3, R, RB>(__VA_ARGS__); break; \
  case 0 * 8 + 4: F<0, 4, R, RB>(__VA_ARGS__); break; \
  case 1 * 8 + 2: F<1, 2, R, RB>(__VA_ARGS__); break; \
  case 1 * 8 + 3: F<1, 3, R, RB>(__VA_ARGS__); break; \
  case 1 * 8 + 4: F<1, 4, R, RB>(__VA_ARGS__); break; \
  case 2 * 8 + 3: F<2, 3, R, RB>(__VA_ARGS__); break; \
  case 2 * 8 + 4: F<2, 4, R, RB>(__VA_ARGS__); break; \
  case 3 * 8 + 4: F<3, 4, R, RB>(__VA_ARGS__); break;

// Applies one instruction to G groups held by this thread (the dispatch and the coefficient loads
// are shared; the G independent updates interleave).
template <class R, int RB, int G>
__device__ __forceinline__ void apply_instr(const Instr& in, Regs<R, RB>* v, const R* __restrict__ coef, uint32_t tile,
                                            const R* tcoef, const uint32_t* grp) {
  const R* c = coef + 2 * size_t(in.coef);
  switch (in.op) {
    case OP_D1G:
      switch (in.a) {
        case 0: for (int g = 0; g < G; ++g) gd1g<0, R, RB>(v[g], c, in.b, grp[g]); break;
        case 1: for (int g = 0; g < G; ++g) gd1g<1, R, RB>(v[g], c, in.b, grp[g]); break;
        case 2: for (int g = 0; g < G; ++g) gd1g<2, R, RB>(v[g], c, in.b, grp[g]); break;
        case 3: for (int g = 0; g < G; ++g) gd1g<3, R, RB>(v[g], c, in.b, grp[g]); break;
        case 4: for (int g = 0; g < G; ++g) gd1g<4, R, RB>(v[g], c, in.b, grp[g]); break;
      }
      break;
    case OP_DTAB:
      for (int g = 0; g < G; ++g) gtab<R, RB>(v[g], c);
      break;
    case OP_1QR:
      switch (in.a) {
        case 0: for (int g = 0; g < G; ++g) g1qs<0, R, RB, false>(v[g], c); break;
        case 1: for (int g = 0; g < G; ++g) g1qs<1, R, RB, false>(v[g], c); break;
        case 2: for (int g = 0; g < G; ++g) g1qs<2, R, RB, false>(v[g], c); break;
        case 3: for (int g = 0; g < G; ++g) g1qs<3, R, RB, false>(v[g], c); break;
        case 4: for (int g = 0; g < G; ++g) g1qs<4, R, RB, false>(v[g], c); break;
      }
      break;
    case OP_1QX:
      switch (in.a) {
        case 0: for (int g = 0; g < G; ++g) g1qs<0, R, RB, true>(v[g], c); break;
        case 1: for (int g = 0; g < G; ++g) g1qs<1, R, RB, true>(v[g], c); break;
        case 2: for (int g = 0; g < G; ++g) g1qs<2, R, RB, true>(v[g], c); break;
        case 3: for (int g = 0; g < G; ++g) g1qs<3, R, RB, true>(v[g], c); break;
        case 4: for (int g = 0; g < G; ++g) g1qs<4, R, RB, true>(v[g], c); break;
      }
      break;
    case OP_D1P: {
      c = tcoef + kTphSlotR * in.coef;
      switch (in.a) {
        case 0: for (int g = 0; g < G; ++g) gd1<0, R, RB>(v[g], c); break;
        case 1: for (int g = 0; g < G; ++g) gd1<1, R, RB>(v[g], c); break;
        case 2: for (int g = 0; g < G; ++g) gd1<2, R, RB>(v[g], c); break;
        case 3: for (int g = 0; g < G; ++g) gd1<3, R, RB>(v[g], c); break;
        case 4: for (int g = 0; g < G; ++g) gd1<4, R, RB>(v[g], c); break;
      }
      break;
    }
    case OP_DTP: {
      c = tcoef + kTphSlotR * in.coef;
      const R pr = c[0], pi = c[1];
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int s = 0; s < (1 << RB); ++s) {
          const R xr = v[g].re(s), xi = v[g].im(s);
          v[g].re(s) = fma(pr, xr, -pi * xi);
          v[g].im(s) = fma(pr, xi, pi * xr);
        }
      break;
    }
    case OP_D1T: {
      // two coefficient blocks (tile bit 0 / 1) in the layout of OP_D1
      constexpr int blk = std::is_same<R, float>::value ? 6 : 2;  // complex entries per block
      c += 2 * blk * ((tile >> in.b) & 1u);
      switch (in.a) {
        case 0: for (int g = 0; g < G; ++g) gd1<0, R, RB>(v[g], c); break;
        case 1: for (int g = 0; g < G; ++g) gd1<1, R, RB>(v[g], c); break;
        case 2: for (int g = 0; g < G; ++g) gd1<2, R, RB>(v[g], c); break;
        case 3: for (int g = 0; g < G; ++g) gd1<3, R, RB>(v[g], c); break;
        case 4: for (int g = 0; g < G; ++g) gd1<4, R, RB>(v[g], c); break;
      }
      break;
    }
    case OP_DT: {
      const uint32_t nb = in.b >> 16;
      uint32_t idx = (tile >> (in.b & 255u)) & 1u;
      if (nb == 2) idx |= ((tile >> ((in.b >> 8) & 255u)) & 1u) << 1;
      const R pr = c[2 * idx], pi = c[2 * idx + 1];
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int s = 0; s < (1 << RB); ++s) {
          const R xr = v[g].re(s), xi = v[g].im(s);
          v[g].re(s) = fma(pr, xr, -pi * xi);
          v[g].im(s) = fma(pr, xi, pi * xr);
        }
      break;
    }
    case OP_1Q:
      switch (in.a) {
        case 0: for (int g = 0; g < G; ++g) g1q<0, R, RB>(v[g], c); break;
        case 1: for (int g = 0; g < G; ++g) g1q<1, R, RB>(v[g], c); break;
        case 2: for (int g = 0; g < G; ++g) g1q<2, R, RB>(v[g], c); break;
        case 3: for (int g = 0; g < G; ++g) g1q<3, R, RB>(v[g], c); break;
        case 4: for (int g = 0; g < G; ++g) g1q<4, R, RB>(v[g], c); break;
      }
      break;
    case OP_D1:
      switch (in.a) {
        case 0: for (int g = 0; g < G; ++g) gd1<0, R, RB>(v[g], c); break;
        case 1: for (int g = 0; g < G; ++g) gd1<1, R, RB>(v[g], c); break;
        case 2: for (int g = 0; g < G; ++g) gd1<2, R, RB>(v[g], c); break;
        case 3: for (int g = 0; g < G; ++g) gd1<3, R, RB>(v[g], c); break;
        case 4: for (int g = 0; g < G; ++g) gd1<4, R, RB>(v[g], c); break;
      }
      break;
    case OP_CX: {
      const uint32_t lo = min(in.a, in.b), hi = max(in.a, in.b);
      const bool fwd = in.a < in.b;  // the control is the lower register bit
      switch (lo * 8 + hi) {
#define QSVB_CX_CASE(J, K)       \
  case J * 8 + K:                \
    for (int g = 0; g < G; ++g)       \
      if (fwd) gcx<J, K, R, RB>(v[g]); \
      else gcx<K, J, R, RB>(v[g]);     \
    break;
        QSVB_CX_CASE(0, 1)
        QSVB_CX_CASE(0, 2)
        QSVB_CX_CASE(0, 3)
        QSVB_CX_CASE(0, 4)
        QSVB_CX_CASE(1, 2)
        QSVB_CX_CASE(1, 3)
        QSVB_CX_CASE(1, 4)
        QSVB_CX_CASE(2, 3)
        QSVB_CX_CASE(2, 4)
        QSVB_CX_CASE(3, 4)
#undef QSVB_CX_CASE
      }
      break;
    }
    case OP_2Q:
      for (int g = 0; g < G; ++g) switch (in.a * 8 + in.b) { QSVB_PAIR_CASES(g2q, v[g], c) }
      break;
    case OP_D2:
      for (int g = 0; g < G; ++g) switch (in.a * 8 + in.b) { QSVB_PAIR_CASES(gd2, v[g], c) }
      break;
  }
}

// One register phase for G groups of this thread: load 2^r amplitudes per group from the swizzled
// tile, apply the phase's instructions, store them back.
template <class R, int RB, int G>
__device__ __forceinline__ void phase_groups(const uint32_t* grp, const PhaseDev& D, const uint32_t* rp, R* xr, R* xi,
                                             const Instr* pprog, uint32_t kbeg, uint32_t kend, const R* pcoef,
                                             uint32_t tile, const R* tcoef) {
  constexpr int NV = 1 << RB;
  const uint32_t r = D.r;
  uint32_t p0[G];
  Regs<R, RB> v[G];
#pragma unroll
  for (int g = 0; g < G; ++g) p0[g] = uint32_t(D.lo[grp[g] & 31u]) ^ uint32_t(D.hi[grp[g] >> 5]);
  if (r == uint32_t(RB)) {  // full register tile (every pass with at least RB local qubits)
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int s = 0; s < NV; ++s) {
        uint32_t off = p0[g];
#pragma unroll
        for (int j = 0; j < RB; ++j)
          if (s & (1 << j)) off ^= rp[j];
        v[g].re(s) = xr[off];
        v[g].im(s) = xi[off];
      }
  } else {
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int s = 0; s < NV; ++s) {
        if (uint32_t(s) >> r) continue;
        uint32_t off = p0[g];
#pragma unroll
        for (int j = 0; j < RB; ++j)
          if (s & (1 << j)) off ^= rp[j];
        v[g].re(s) = xr[off];
        v[g].im(s) = xi[off];
      }
  }
  for (uint32_t kk = kbeg; kk < kend; ++kk) apply_instr<R, RB, G>(pprog[kk], v, pcoef, tile, tcoef, grp);
  if (r == uint32_t(RB)) {
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int s = 0; s < NV; ++s) {
        uint32_t off = p0[g];
#pragma unroll
        for (int j = 0; j < RB; ++j)
          if (s & (1 << j)) off ^= rp[j];
        xr[off] = v[g].re(s);
        xi[off] = v[g].im(s);
      }
  } else {
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int s = 0; s < NV; ++s) {
        if (uint32_t(s) >> r) continue;
        uint32_t off = p0[g];
#pragma unroll
        for (int j = 0; j < RB; ++j)
          if (s & (1 << j)) off ^= rp[j];
        xr[off] = v[g].re(s);
        xi[off] = v[g].im(s);
      }
  }
}

// HI: entries of the address and swizzle tables (2^(lbits - 5) and 2^(lbits - W) at most); tile
// sweeps take a smaller table, which leaves room for one more block per SM.
template <class R, int RB, int W, int NT, int MINB = 1, int GP = 1, int HI = kMaxHi>
__global__ void __launch_bounds__(NT, MINB)
    k_batch(const Item* __restrict__ items, uint32_t nitems, const PassDev* __restrict__ passes,
            const PhaseDev* __restrict__ phases, const Instr* __restrict__ prog, const R* __restrict__ coef,
            R* __restrict__ sre, R* __restrict__ sim, double* __restrict__ probs, double* __restrict__ zpart,
            uint32_t* __restrict__ done, uint32_t* __restrict__ queue, int* __restrict__ err, uint32_t lbits,
            long long* __restrict__ prof, uint32_t fixed, const long long* __restrict__ wait_budget) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  R* xr = reinterpret_cast<R*>(smem_raw);
  R* xi = xr + (size_t(1) << lbits);  // every pass has nlocal <= lbits
  uint8_t* stage = reinterpret_cast<uint8_t*>(xi + (size_t(1) << lbits));  // the pass's program
  // per-tile phase coefficients (tile sweeps; sits right after the program staging area)
  R* tcoef = reinterpret_cast<R*>(stage + (fixed ? kTileStageBytes : kStageBytes));
  __shared__ uint64_t s_gaddr[HI];
  __shared__ uint16_t s_swz[HI];
  __shared__ uint32_t s_item;
  __shared__ double s_red[NT / 32];
  __shared__ int s_ok;
  const int tid = threadIdx.x;
  // clock64 cycles one dependency wait may take before the run is failed (device memory, so that a
  // captured graph picks up a changed value; nullptr: the default)
  const long long budget = wait_budget != nullptr ? *wait_budget : kSpinBudget;
  // swizzle table over the index bits above W
  for (uint32_t h = tid; h < (1u << (lbits - W)); h += NT) {
    uint32_t v = 0;
    for (int i = 0; i < int(lbits) - W; ++i)
      if ((h >> i) & 1u) v ^= swz_col(W + i, W);
    if (QSVB_BC(h < uint32_t(HI), err)) s_swz[h] = uint16_t(v);
  }
  long long t_wait = 0, t_fill = 0, t_gates = 0, t_out = 0, n_items = 0, t_mark = prof ? clock64() : 0;
  uint32_t staged_pass = ~0u;
  // fixed != 0: one pass (passes[0]) over one state, tile i handled by block i mod grid, no queue
  uint32_t iter = 0;
  while (true) {
    if (!fixed && tid == 0) s_item = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t it = fixed ? blockIdx.x + (iter++) * gridDim.x : s_item;
    if (it >= nitems) break;
    const Item item = fixed ? Item{0u, it} : items[it];
    const PassDev& P = passes[item.pass];
    const uint32_t L = P.nlocal, T = 1u << L;
    [[maybe_unused]] const uint64_t gsize = 1ull << (L + P.nnon);  // the circuit's amplitudes (checked builds)
    if (tid == 0) {
      int ok = *reinterpret_cast<volatile int*>(err) == 0;
      if (ok && P.prev != ~0u) {
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> d(done[P.prev]);
        const uint32_t need = passes[P.prev].ntiles;
        if (d.load(cuda::memory_order_acquire) < need) {
          const long long t0 = clock64();
          while (d.load(cuda::memory_order_acquire) < need) {
            if (clock64() - t0 > budget) {
              ok = 0;
              atomicOr(err, kErrTimeout);
              break;
            }
            if (*reinterpret_cast<volatile int*>(err)) {  // an earlier wait gave up: abandon fast
              ok = 0;
              break;
            }
            __nanosleep(256);
          }
        }
      }
      s_ok = ok;
    }
    // global offset of each value of the local index bits above bit 4 (local positions 0..4 are
    // state bits 0..4, contiguous in memory)
    const uint32_t nhi = L > 5 ? L - 5 : 0;
    {
      uint64_t base = 0;
      for (uint32_t j = 0; j < P.nnon; ++j) base |= uint64_t((item.tile >> j) & 1u) << P.nonlocal[j];
      for (uint32_t h = tid; h < (1u << nhi); h += NT) {
        uint64_t a = base;
        for (uint32_t j = 0; j < nhi; ++j) a |= uint64_t((h >> j) & 1u) << P.local[5 + j];
        if (QSVB_BC(h < uint32_t(HI), err)) s_gaddr[h] = a;
      }
    }
    __syncthreads();
    if (prof) t_wait += clock64() - t_mark, t_mark = clock64(), ++n_items;
    if (!s_ok) continue;
    // the pass's instructions, phases and coefficients into shared memory (kept while the next
    // item is a tile of the same pass), overlapped with the tile fill
    const uint32_t ph_bytes = P.prog_len * uint32_t(sizeof(Instr));
    const uint32_t co_bytes = (ph_bytes + P.nphase * uint32_t(sizeof(PhaseDev)) + 7u) & ~7u;
    if (P.staged && staged_pass != item.pass &&
        QSVB_BC(co_bytes + P.ncoef * 2u * uint32_t(sizeof(R)) <= (fixed ? kTileStageBytes : kStageBytes), err)) {
      const uint32_t* src0 = reinterpret_cast<const uint32_t*>(prog + P.prog_off);
      const uint32_t* src1 = reinterpret_cast<const uint32_t*>(phases + P.phase_off);
      const uint32_t* src2 = reinterpret_cast<const uint32_t*>(coef + 2 * size_t(P.coef_off));
      uint32_t* dst = reinterpret_cast<uint32_t*>(stage);
      const uint32_t n0 = ph_bytes / 4, n1 = P.nphase * uint32_t(sizeof(PhaseDev)) / 4;
      const uint32_t n2 = P.ncoef * 2u * uint32_t(sizeof(R)) / 4;
      for (uint32_t w = tid; w < n0; w += NT) cp_async_elem(dst + w, src0 + w);
      for (uint32_t w = tid; w < n1; w += NT) cp_async_elem(dst + n0 + w, src1 + w);
      for (uint32_t w = tid; w < n2; w += NT) cp_async_elem(dst + co_bytes / 4 + w, src2 + w);
    }
    staged_pass = P.staged ? item.pass : ~0u;
    const Instr* pprog = P.staged ? reinterpret_cast<const Instr*>(stage) : prog + P.prog_off;
    const PhaseDev* pph = P.staged ? reinterpret_cast<const PhaseDev*>(stage + ph_bytes) : phases + P.phase_off;
    const R* pcoef = P.staged ? reinterpret_cast<const R*>(stage + co_bytes) : coef + 2 * size_t(P.coef_off);
    const uint32_t lowmask = L >= 5 ? 31u : (T - 1u);
    R* gre = sre + P.state_off;
    R* gim = sim + P.state_off;
    if (P.first) {
      for (uint32_t x = tid; x < T; x += NT) {
        xr[x] = R(0);
        xi[x] = R(0);
      }
      __syncthreads();
      if (tid == 0 && item.tile == 0) xr[0] = R(1);  // the swizzle maps 0 to 0
    } else if (L >= 5 && sizeof(R) != 8) {
      // 16-byte loads of contiguous amplitudes (a run of 32 shares its global offset), several in
      // flight per thread, then scattered through the swizzle (it only flips bits below W, so the
      // VN amplitudes of a vector land at y ^ e). complex128 takes the per-element cp.async path
      // below instead: the whole tile in flight at once with no registers held (measured 3-4 %
      // faster for tile sweeps and 2 % for batches; 1.5-4 % slower for complex64)
      using VT = typename Vec16<R>::T;
      constexpr int VN = Vec16<R>::N, UNR = 4;
      for (uint32_t xb = tid * VN; xb < T; xb += NT * VN * UNR) {
        VT vr[UNR], vi[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
          const uint32_t x = xb + uint32_t(u) * NT * VN;
          if (x < T) {
            const uint64_t a = s_gaddr[x >> 5] | (x & 31u);
            if (!QSVB_BC(a + VN <= gsize, err)) continue;
            vr[u] = __ldcg(reinterpret_cast<const VT*>(gre + a));
            vi[u] = __ldcg(reinterpret_cast<const VT*>(gim + a));
          }
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
          const uint32_t x = xb + uint32_t(u) * NT * VN;
          if (x < T) {
            const uint32_t y = x ^ s_swz[x >> W];
            if (!QSVB_BC((y | uint32_t(VN - 1)) < T, err)) continue;
#pragma unroll
            for (int e = 0; e < VN; ++e) {
              xr[y ^ uint32_t(e)] = Vec16<R>::get(vr[u], e);
              xi[y ^ uint32_t(e)] = Vec16<R>::get(vi[u], e);
            }
          }
        }
      }
    } else {
      for (uint32_t x = tid; x < T; x += NT) {
        const uint64_t a = s_gaddr[x >> 5] | (x & lowmask);
        const uint32_t y = x ^ s_swz[x >> W];
        if (!QSVB_BC(a < gsize && y < T, err)) continue;
        cp_async_elem(xr + y, gre + a);
        cp_async_elem(xi + y, gim + a);
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    if (P.tph_n) {
      // phase sums over the tile bits, one slot per operation: D1 blocks (the 0 and 1 sides of a
      // register bit) or a single complex factor
      const uint8_t* tb = reinterpret_cast<const uint8_t*>(&P) + P.tph_off;
      const uint32_t* offs = reinterpret_cast<const uint32_t*>(tb);
      const double* dd = reinterpret_cast<const double*>(tb + ((4 * P.tph_n + 7) & ~7u));
      for (uint32_t i = tid; i < P.tph_n; i += NT) {
        // unit factors multiplied in FP64: no sin/cos per tile
        const double* d = dd + offs[i];
        const int type = int(d[0]), m = int(d[5]);
        double z0r = d[1], z0i = d[2], z1r = d[3], z1i = d[4];
        for (int t = 0; t < m; ++t) {
          const double* term = d + 6 + 6 * t;
          const uint32_t k = uint32_t(term[0]), l = uint32_t(term[1]);
          if (((item.tile >> k) & (item.tile >> l) & 1u) == 0u) continue;
          double r = z0r * term[2] - z0i * term[3];
          z0i = z0r * term[3] + z0i * term[2];
          z0r = r;
          if (type == 1) {
            r = z1r * term[4] - z1i * term[5];
            z1i = z1r * term[5] + z1i * term[4];
            z1r = r;
          }
        }
        const double c0 = z0r, s0 = z0i, c1 = z1r, s1 = z1i;
        R* o = tcoef + kTphSlotR * i;
        if (type == 2) {
          o[0] = R(c0);
          o[1] = R(s0);
        } else if constexpr (std::is_same<R, float>::value) {
          const bool j0 = d[6 + 6 * m] != 0.0;  // register bit 0: lanes take the two sides
          const float v[3][2] = {{float(c0), float(c1)}, {float(s0), float(s1)}, {float(-s0), float(-s1)}};
          if (j0) {
            for (int rep = 0; rep < 2; ++rep)
              for (int e = 0; e < 3; ++e) {
                o[6 * rep + 2 * e] = v[e][0];
                o[6 * rep + 2 * e + 1] = v[e][1];
              }
          } else {
            const float w[6] = {float(c0), float(s0), float(-s0), float(c1), float(s1), float(-s1)};
            for (int e = 0; e < 6; ++e) o[2 * e] = o[2 * e + 1] = w[e];
          }
        } else {
          o[0] = R(c0);
          o[1] = R(s0);
          o[2] = R(c1);
          o[3] = R(s1);
        }
      }
      __syncthreads();
    }
    if (prof) t_fill += clock64() - t_mark, t_mark = clock64();
    // register phases: each group of 2^r amplitudes (fixed non-register bits) is loaded into one
    // thread's registers, takes all of the phase's gates there, and is written back
    uint32_t k = 0;
    while (k < P.prog_len) {
      const PhaseDev& D = pph[pprog[k].coef];
      const uint32_t nt = D.nt;
      const uint32_t kbeg = k + 1, kend = kbeg + D.ninstr;
      uint32_t rp[RB];
#pragma unroll
      for (int j = 0; j < RB; ++j) rp[j] = D.rphys[j];
      // (checked builds) a group's offsets are XORs of these and of its two table entries, so each
      // below T keeps every offset in the tile
      bool rp_ok = true;
#pragma unroll
      for (int j = 0; j < RB; ++j) rp_ok = rp_ok && (uint32_t(j) >= D.r || QSVB_BC(rp[j] < T, err));  // bits in use
      auto grp_ok = [&](uint32_t gi) { return rp_ok && QSVB_BC((uint32_t(D.lo[gi & 31u]) ^ uint32_t(D.hi[gi >> 5])) < T, err); };
      // two groups at a time where the thread has two (independent updates interleave), then one
      const uint32_t ngrp = 1u << nt;
      uint32_t grp = tid;
      if constexpr (GP == 2) {
        for (; grp + NT < ngrp; grp += 2 * NT) {
          const uint32_t gg[2] = {grp, grp + NT};
          if (grp_ok(gg[0]) && grp_ok(gg[1]))
            phase_groups<R, RB, 2>(gg, D, rp, xr, xi, pprog, kbeg, kend, pcoef, item.tile, tcoef);
        }
      }
      for (; grp < ngrp; grp += NT) {
        const uint32_t gg[1] = {grp};
        if (grp_ok(gg[0])) phase_groups<R, RB, 1>(gg, D, rp, xr, xi, pprog, kbeg, kend, pcoef, item.tile, tcoef);
      }
      k = kend;
      __syncthreads();
    }
    if (prof) t_gates += clock64() - t_mark, t_mark = clock64();
    if (P.last) {
      // FP64 probabilities and the <Z_0> partial (state bit 0 is local position 0)
      double z = 0.0;
      double* pout = probs + P.prob_off;
      for (uint32_t x = tid; x < T; x += NT) {
        const uint32_t y = x ^ s_swz[x >> W];
        const uint64_t pa = s_gaddr[x >> 5] | (x & lowmask);
        if (!QSVB_BC(pa < gsize && y < T, err)) continue;
        const double p = double(xr[y]) * double(xr[y]) + double(xi[y]) * double(xi[y]);
        __stcs(pout + pa, p);
        z += (x & 1u) ? -p : p;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
      if ((tid & 31) == 0) s_red[tid >> 5] = z;
      __syncthreads();
      if (tid == 0) {
        double s = 0.0;
        for (int w = 0; w < NT / 32; ++w) s += s_red[w];
        zpart[P.zslot + item.tile] = s;
      }
    } else if (L >= 5) {
      using VT = typename Vec16<R>::T;
      constexpr int VN = Vec16<R>::N;
      for (uint32_t x = tid * VN; x < T; x += NT * VN) {
        const uint64_t a = s_gaddr[x >> 5] | (x & 31u);
        const uint32_t y = x ^ s_swz[x >> W];
        if (!QSVB_BC(a + VN <= gsize && (y | uint32_t(VN - 1)) < T, err)) continue;
        VT vr, vi;
#pragma unroll
        for (int e = 0; e < VN; ++e) {
          Vec16<R>::set(vr, e, xr[y ^ uint32_t(e)]);
          Vec16<R>::set(vi, e, xi[y ^ uint32_t(e)]);
        }
        __stcg(reinterpret_cast<VT*>(gre + a), vr);
        __stcg(reinterpret_cast<VT*>(gim + a), vi);
      }
    } else {
      for (uint32_t x = tid; x < T; x += NT) {
        const uint64_t a = s_gaddr[x >> 5] | (x & lowmask);
        const uint32_t y = x ^ s_swz[x >> W];
        if (!QSVB_BC(a < gsize && y < T, err)) continue;
        __stcg(gre + a, xr[y]);
        __stcg(gim + a, xi[y]);
      }
    }
    __syncthreads();
    if (tid == 0 && !fixed) {
      __threadfence();
      cuda::atomic_ref<uint32_t, cuda::thread_scope_device> d(done[item.pass]);
      d.fetch_add(1u, cuda::memory_order_release);
    }
    if (prof) t_out += clock64() - t_mark, t_mark = clock64();
  }
  if (prof && tid == 0) {
    long long* o = prof + 5 * blockIdx.x;
    o[0] = t_wait;
    o[1] = t_fill;
    o[2] = t_gates;
    o[3] = t_out;
    o[4] = n_items;
  }
}

__global__ void k_batch_z0(const double* __restrict__ zpart, const uint64_t* __restrict__ zoff,
                           const uint32_t* __restrict__ zcnt, uint32_t ncirc, double* __restrict__ z0) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncirc) return;
  double s = 0.0;
  for (uint32_t t = 0; t < zcnt[c]; ++t) s += zpart[zoff[c] + t];
  z0[c] = s;
}

// ------------------------------------------------------------------------------------ host plan
struct HostGate {
  uint32_t m;
  uint32_t q[2];
  std::vector<cd> a;
};

enum LKind : uint32_t {
  LK_1Q = OP_1Q, LK_D1 = OP_D1, LK_CX = OP_CX, LK_2Q = OP_2Q, LK_D2 = OP_D2, LK_D1T = OP_D1T, LK_DT = OP_DT,
  LK_D1P = OP_D1P, LK_DTP = OP_DTP
};

// A phase sum evaluated once per tile (type 1: the two sides of one local qubit, linear in tile
// bits; type 2: one factor, quadratic in tile bits). Angles in FP64.
struct TphOp {
  int type = 1;
  double c0 = 0, c1 = 0;
  std::vector<std::array<double, 3>> terms;  // type 1: (bit, d0, d1); type 2: (bit k, bit l, angle)
  bool j0 = false;                           // type 1: lives on register bit 0 of its phase
};

struct LGate {  // a gate on local positions
  uint32_t kind;
  uint32_t p[2];
  const HostGate* g;
  // LK_D1T: t[0] = tile bit, swapq = the local qubit is the gate's second qubit (entry bit 1);
  // LK_DT: nt tile bits t[0] (entry bit 0) and t[1] (entry bit 1)
  uint32_t t[2] = {0, 0};
  uint32_t nt = 0;
  bool swapq = false;
};

uint32_t lgate_mask(const LGate& g) {
  switch (g.kind) {
    case LK_1Q:
    case LK_D1:
    case LK_D1P:
    case LK_D1T: return 1u << g.p[0];
    case LK_DT:
    case LK_DTP: return 0u;
    default: return (1u << g.p[0]) | (1u << g.p[1]);
  }
}

bool lgate_diag(const LGate& g) {
  return g.kind == LK_D1 || g.kind == LK_D2 || g.kind == LK_D1T || g.kind == LK_DT || g.kind == LK_D1P ||
         g.kind == LK_DTP;
}

std::vector<HostGate> fuse_single_qubit_runs(const qsvb_circuit& c) {
  // consecutive gates on the same single qubit are composed (exactly, in FP64); the rest stays
  std::vector<HostGate> out;
  std::vector<int> open1q(c.n_qubits, -1);  // index in `out` of the open 1q gate on each qubit
  for (size_t i = 0; i < c.n_gates; ++i) {
    const qsvb_gate& g = c.gates[i];
    QSVB_REQUIRE(g.n_qubits <= 2, "batched circuits take 1- and 2-qubit gates (gate " + std::to_string(i) + ")");
    HostGate h;
    h.m = g.n_qubits;
    h.q[0] = g.qubits[0];
    h.q[1] = h.m == 2 ? g.qubits[1] : 0u;
    const size_t d = size_t(1) << h.m;
    h.a.resize(d * d);
    for (size_t k = 0; k < d * d; ++k) h.a[k] = cd(g.matrix[2 * k], g.matrix[2 * k + 1]);
    if (h.m == 1 && open1q[h.q[0]] >= 0) {
      HostGate& o = out[size_t(open1q[h.q[0]])];
      std::vector<cd> r(4);
      for (int x = 0; x < 2; ++x)
        for (int y = 0; y < 2; ++y) r[x * 2 + y] = h.a[x * 2 + 0] * o.a[0 * 2 + y] + h.a[x * 2 + 1] * o.a[1 * 2 + y];
      o.a = r;
      continue;
    }
    for (uint32_t j = 0; j < h.m; ++j) open1q[h.q[j]] = -1;
    out.push_back(std::move(h));
    if (out.back().m == 1) open1q[out.back().q[0]] = int(out.size() - 1);
  }
  return out;
}

uint32_t gate_kind(const HostGate& g) {
  const size_t d = size_t(1) << g.m;
  bool diag = true;
  for (size_t r = 0; r < d; ++r)
    for (size_t c = 0; c < d; ++c)
      if (r != c && g.a[r * d + c] != cd(0, 0)) diag = false;
  if (g.m == 1) return diag ? LK_D1 : LK_1Q;
  if (diag) return LK_D2;
  static const double cx[16] = {1, 0, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0};
  bool is_cx = true;
  for (int k = 0; k < 16; ++k) is_cx = is_cx && g.a[size_t(k)] == cd(cx[k], 0);
  return is_cx ? LK_CX : LK_2Q;
}

}  // namespace

struct BatchPlan {
  int dtype = 0;
  uint32_t local_bits = 14, rb = 5, swz_w = 5;
  uint32_t ncirc = 0;
  std::vector<PassDev> passes;
  std::vector<PhaseDev> phases;
  std::vector<Instr> prog;
  std::vector<double> coef;  // complex entries as (re, im) pairs in FP64
  std::vector<Item> items;
  std::vector<uint64_t> prob_off, zoff;
  std::vector<uint32_t> zcnt, nq;
  uint64_t state_amps = 0, prob_total = 0, zslots = 0;
  qsvb_plan_stats stats{};
};

namespace {

void push_coef(BatchPlan& bp, const cd& v) {
  bp.coef.push_back(v.real());
  bp.coef.push_back(v.imag());
}

// A 2x2 gate whose entries are each real or imaginary: 1 for a real matrix [[a, b], [c, d]], 2 for
// [[a, i b], [i c, d]] with a..d real (k = a, b, c, d), 0 otherwise. Parts within 1e-15 of the
// largest entry's magnitude count as zero.
int split_form(const std::vector<cd>& u, double k[4]) {
  double mx = 0;
  for (int e = 0; e < 4; ++e) mx = std::max(mx, std::abs(u[e]));
  const double tol = 1e-15 * mx;
  auto z = [&](double x) { return std::abs(x) <= tol; };
  if (z(u[0].imag()) && z(u[1].imag()) && z(u[2].imag()) && z(u[3].imag())) {
    for (int e = 0; e < 4; ++e) k[e] = u[e].real();
    return 1;
  }
  if (z(u[0].imag()) && z(u[3].imag()) && z(u[1].real()) && z(u[2].real())) {
    k[0] = u[0].real();
    k[1] = u[1].imag();
    k[2] = u[2].imag();
    k[3] = u[3].real();
    return 2;
  }
  return 0;
}

// Splits a pass's gates into register phases and appends them to the plan's program.
void emit_phases(BatchPlan& bp, const std::vector<LGate>& G, uint32_t nlocal, std::vector<TphOp>* tph = nullptr) {
  // phase and coefficient indices are relative to the pass (its program is staged as one block)
  const size_t phase_base = bp.phases.size(), coef_base = bp.coef.size() / 2;
  const uint32_t rb = std::min(bp.rb, nlocal);
  const uint32_t W = bp.swz_w;
  const uint32_t all = (1u << nlocal) - 1u;
  std::vector<char> done(G.size(), 0);
  size_t first = 0;
  std::vector<size_t> taken;
  while (true) {
    while (first < G.size() && done[first]) ++first;
    if (first == G.size()) break;
    // blocked: positions of skipped non-diagonal gates; dblocked: of skipped diagonal gates (a
    // diagonal gate may still pass those)
    uint32_t Rm = 0, blocked = 0, dblocked = 0;
    taken.clear();
    for (size_t i = first; i < G.size(); ++i) {
      if (done[i]) continue;
      const LGate& g = G[i];
      const uint32_t m = lgate_mask(g);
      const bool diag = lgate_diag(g);
      if ((m & blocked) == 0 && (diag || (m & dblocked) == 0) && uint32_t(__builtin_popcount(Rm | m)) <= rb) {
        Rm |= m;
        done[i] = 1;
        taken.push_back(i);
      } else if (g.kind == LK_D2 && (m & blocked) == 0 && __builtin_popcount(m & Rm) == 1) {
        // a 2-qubit diagonal with one qubit in the registers: the other is a group-index bit of
        // this phase, so each thread applies the entries its group selects (OP_D1G)
        done[i] = 1;
        taken.push_back(i);
      } else if (diag) {
        dblocked |= m;
      } else {
        blocked |= m;
      }
      const bool full = uint32_t(__builtin_popcount(Rm)) == rb;
      if ((blocked | dblocked) == all || (full && (Rm & ~(blocked | dblocked)) == 0)) break;
    }
    for (uint32_t p = 0; p < nlocal && uint32_t(__builtin_popcount(Rm)) < rb; ++p) Rm |= 1u << p;
    // register bits: the phase's local positions in ascending order
    int regbit[32];
    uint32_t nr = 0;
    PhaseDev D{};
    for (uint32_t p = 0; p < nlocal; ++p) {
      regbit[p] = -1;
      if ((Rm >> p) & 1u) {
        regbit[p] = int(nr);
        D.rphys[nr++] = (1u << p) ^ swz_col(int(p), int(W));
      }
    }
    D.r = nr;
    // lanes: non-register positions whose bank bits span the W bank-selecting bits
    std::vector<uint32_t> nonr, lanes;
    for (uint32_t p = 0; p < nlocal; ++p)
      if (!((Rm >> p) & 1u)) nonr.push_back(p);
    const size_t nlanes = std::min<size_t>(5, nonr.size());
    uint32_t basis[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // GF(2) elimination keyed by leading bit
    std::vector<char> used(nonr.size(), 0);
    for (size_t i = 0; i < nonr.size() && lanes.size() < nlanes; ++i) {
      const uint32_t p = nonr[i];
      uint32_t v = ((1u << p) ^ swz_col(int(p), int(W))) & ((1u << W) - 1u);
      for (int b = int(W) - 1; b >= 0 && v; --b) {
        if (!((v >> b) & 1u)) continue;
        if (basis[b]) {
          v ^= basis[b];
        } else {
          basis[b] = v;
          break;
        }
      }
      if (v) {
        lanes.push_back(p);
        used[i] = 1;
      }
    }
    for (size_t i = 0; i < nonr.size() && lanes.size() < nlanes; ++i)
      if (!used[i]) {
        lanes.push_back(nonr[i]);
        used[i] = 1;
      }
    for (size_t i = 0; i < nonr.size(); ++i)
      if (!used[i]) lanes.push_back(nonr[i]);
    D.nt = uint32_t(nonr.size());
    QSVB_REQUIRE(D.nt <= 10, "register phase with more than 2^10 groups");
    int gbit_of[32];  // local position -> its bit in the group index (-1: a register bit)
    for (int q = 0; q < 32; ++q) gbit_of[q] = -1;
    for (size_t i = 0; i < lanes.size(); ++i) gbit_of[lanes[i]] = int(i);
    // group index bits -> local positions (lanes first), as swizzled offsets: the swizzle is
    // linear, so the offset of a group is the XOR of the offsets of its bits
    auto phys_of = [&](uint32_t pos) { return (1u << pos) ^ swz_col(int(pos), int(W)); };
    for (uint32_t g = 0; g < 32; ++g) {
      uint32_t lo = 0, hi = 0;
      for (uint32_t i = 0; i < 5 && i < D.nt; ++i)
        if ((g >> i) & 1u) lo ^= phys_of(lanes[i]);
      for (uint32_t i = 5; i < 10 && i < D.nt; ++i)
        if ((g >> (i - 5)) & 1u) hi ^= phys_of(lanes[i]);
      D.lo[g] = uint16_t(lo);
      D.hi[g] = uint16_t(hi);
    }
    const size_t phase_idx = bp.phases.size(), phase_pc = bp.prog.size();
    bp.prog.push_back(Instr{OP_PHASE, 0, 0, uint32_t(bp.phases.size() - phase_base)});
    bp.phases.push_back(D);
    // Emission. Non-diagonal operations keep their order (1-qubit gates of split form as OP_1QR /
    // OP_1QX).
    // Diagonal factors on register bits (LK_D1, LK_D2) are multiplied into per-slot tables: a factor
    // may sit anywhere between the last non-diagonal operation on its bits before it and the first
    // one after it, and the tables go where the fewest points cover every factor's range (interval
    // stabbing, ends first).
    const uint32_t nslot = 1u << bp.rb;
    struct Op {
      const LGate* g;  // nullptr: a split-form 1-qubit gate or group-dependent diagonal on rbit
      uint32_t rbit;
      int form;        // split_form: 1 real, 2 imaginary off-diagonal; 3: OP_D1G (factors gf[gidx])
      double k[4];
      int gidx;
    };
    // group-dependent diagonals on a register bit: (group bit, the 4 entries indexed register bit |
    // group bit << 1), merged per group bit, pending until the next non-diagonal op on that bit
    struct GFac {
      uint32_t gbit;
      cd d[4];
    };
    std::vector<std::vector<GFac>> gfs;
    std::vector<GFac> pend_g[8];
    struct Fac {
      uint32_t rb0, rb1, nb;  // register bits (nb = 1 or 2)
      cd d[4];                // diagonal entries, index bit 0 <-> rb0, bit 1 <-> rb1
      size_t lo, hi;          // allowed slots: before ops[j], lo <= j <= hi
    };
    std::vector<Op> ops;
    std::vector<Fac> facs;
    int last_nd[8] = {-1, -1, -1, -1, -1, -1, -1, -1};  // per register bit: last non-diagonal op
    std::vector<size_t> open_facs;                      // factors whose upper end is not known yet
    auto add_fac = [&](uint32_t rb0, uint32_t rb1, uint32_t nb, const cd* d) {
      Fac f{};
      f.rb0 = rb0;
      f.rb1 = rb1;
      f.nb = nb;
      for (uint32_t e = 0; e < (1u << nb); ++e) f.d[e] = d[e];
      int lo = last_nd[rb0];
      if (nb == 2) lo = std::max(lo, last_nd[rb1]);
      f.lo = size_t(lo + 1);
      f.hi = SIZE_MAX;
      open_facs.push_back(facs.size());
      facs.push_back(f);
    };
    auto flush_g = [&](uint32_t rbit) {
      if (pend_g[rbit].empty()) return;
      std::sort(pend_g[rbit].begin(), pend_g[rbit].end(), [](const GFac& x, const GFac& y) { return x.gbit < y.gbit; });
      gfs.push_back(std::move(pend_g[rbit]));
      pend_g[rbit].clear();
      ops.push_back(Op{nullptr, rbit, 3, {0, 0, 0, 0}, int(gfs.size() - 1)});
    };
    auto add_gfac = [&](uint32_t rbit, uint32_t gbit, const cd* d) {
      for (GFac& f : pend_g[rbit])
        if (f.gbit == gbit) {
          for (int e = 0; e < 4; ++e) f.d[e] *= d[e];
          return;
        }
      GFac f{gbit, {d[0], d[1], d[2], d[3]}};
      pend_g[rbit].push_back(f);
    };
    auto add_nondiag = [&](const Op& op, uint32_t bits) {
      for (uint32_t b = 0; b < 8; ++b)
        if ((bits >> b) & 1u) flush_g(b);
      const size_t idx = ops.size();
      ops.push_back(op);
      for (size_t fi : open_facs) {
        Fac& f = facs[fi];
        const uint32_t fm = (1u << f.rb0) | (f.nb == 2 ? (1u << f.rb1) : 0u);
        if (f.hi == SIZE_MAX && (fm & bits)) f.hi = idx;
      }
      for (uint32_t b = 0; b < 8; ++b)
        if ((bits >> b) & 1u) last_nd[b] = int(idx);
    };
    for (size_t i : taken) {
      const LGate& g = G[i];
      const std::vector<cd>& a = g.g->a;
      if (g.kind == LK_D1) {
        const cd d[2] = {a[0], a[3]};
        add_fac(uint32_t(regbit[g.p[0]]), 0, 1, d);
        continue;
      }
      if (g.kind == LK_D2 && (regbit[g.p[0]] < 0 || regbit[g.p[1]] < 0)) {
        // entry index bit 0 <-> p[0], bit 1 <-> p[1]; OP_D1G wants register bit | group bit << 1
        const bool in0 = regbit[g.p[0]] >= 0;
        const uint32_t pout = in0 ? g.p[1] : g.p[0];
        const cd d[4] = {a[0], a[in0 ? 5 : 10], a[in0 ? 10 : 5], a[15]};
        QSVB_REQUIRE(gbit_of[pout] >= 0, "group-dependent diagonal outside the phase's group bits");
        add_gfac(uint32_t(regbit[in0 ? g.p[0] : g.p[1]]), uint32_t(gbit_of[pout]), d);
        continue;
      }
      if (g.kind == LK_D2) {
        const cd d[4] = {a[0], a[5], a[10], a[15]};
        add_fac(uint32_t(regbit[g.p[0]]), uint32_t(regbit[g.p[1]]), 2, d);
        continue;
      }
      if (g.kind == LK_1Q) {
        // entries each real or imaginary (RY, H, X; RX, Y): half the work of a general 1-qubit gate
        Op op{nullptr, 0, 0, {0, 0, 0, 0}, -1};
        op.form = split_form(a, op.k);
        if (op.form != 0) {
          op.rbit = uint32_t(regbit[g.p[0]]);
          add_nondiag(op, 1u << op.rbit);
          continue;
        }
      }
      uint32_t bits = 0;
      if (!lgate_diag(g)) {
        const uint32_t lm = lgate_mask(g);
        for (uint32_t p = 0; p < nlocal; ++p)
          if (((lm >> p) & 1u) && regbit[p] >= 0) bits |= 1u << regbit[p];
      }
      add_nondiag(Op{&g, 0, 0, {0, 0, 0, 0}, -1}, bits);  // diagonal kinds outside tables constrain nothing
    }
    for (uint32_t b = 0; b < 8; ++b) flush_g(b);
    for (Fac& f : facs)
      if (f.hi == SIZE_MAX) f.hi = ops.size();
    std::vector<size_t> order(facs.size());
    std::iota(order.begin(), order.end(), size_t(0));
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return facs[x].hi < facs[y].hi; });
    std::vector<std::vector<cd>> tables(ops.size() + 1);
    size_t point = SIZE_MAX;
    for (size_t fi : order) {
      const Fac& f = facs[fi];
      if (point == SIZE_MAX || point < f.lo) point = f.hi;
      std::vector<cd>& t = tables[point];
      if (t.empty()) t.assign(nslot, cd(1, 0));
      for (uint32_t s2 = 0; s2 < nslot; ++s2) {
        size_t e = (s2 >> f.rb0) & 1u;
        if (f.nb == 2) e |= size_t((s2 >> f.rb1) & 1u) << 1;
        t[s2] *= f.d[e];
      }
    }
    auto emit_table = [&](const std::vector<cd>& t) {
      const size_t base = bp.coef.size() / 2;
      if (bp.dtype == QSVB_C64) {
        for (uint32_t h = 0; h < nslot / 2; ++h) {
          const cd a0 = t[2 * h], a1 = t[2 * h + 1];
          push_coef(bp, cd(a0.real(), a1.real()));
          push_coef(bp, cd(a0.imag(), a1.imag()));
          push_coef(bp, cd(-a0.imag(), -a1.imag()));
        }
      } else {
        for (uint32_t s2 = 0; s2 < nslot; ++s2) push_coef(bp, t[s2]);
      }
      bp.prog.push_back(Instr{OP_DTAB, 0, 0, uint32_t(base - coef_base)});
    };
    auto emit_group = [&](const Op& op) {
      uint32_t mask = 0;
      const uint32_t base = uint32_t(bp.coef.size() / 2 - coef_base);
      for (const GFac& f : gfs[size_t(op.gidx)]) {
        mask |= 1u << f.gbit;
        for (int e = 0; e < 4; ++e) push_coef(bp, f.d[e]);
      }
      bp.prog.push_back(Instr{OP_D1G, op.rbit, mask, base});
    };
    auto emit_split = [&](const Op& op) {
      Instr in{op.form == 2 ? uint32_t(OP_1QX) : uint32_t(OP_1QR), op.rbit, 0,
               uint32_t(bp.coef.size() / 2 - coef_base)};
      if (bp.dtype == QSVB_C64) {  // pre-broadcast pairs (a, a), (b, b), (c, c), (d, d) [, (-b, -b), (-c, -c)]
        for (int e = 0; e < 4; ++e) push_coef(bp, cd(op.k[e], op.k[e]));
        if (op.form == 2) {
          push_coef(bp, cd(-op.k[1], -op.k[1]));
          push_coef(bp, cd(-op.k[2], -op.k[2]));
        }
      } else {
        push_coef(bp, cd(op.k[0], op.k[1]));
        push_coef(bp, cd(op.k[2], op.k[3]));
      }
      bp.prog.push_back(in);
    };
    auto emit_one = [&](const LGate& g) {
        Instr in{g.kind, uint32_t(regbit[g.p[0]]), 0, uint32_t(bp.coef.size() / 2 - coef_base)};
        const std::vector<cd>& a = g.g->a;
        switch (g.kind) {
          case LK_1Q:
            if (bp.dtype == QSVB_C64) {  // pre-broadcast pairs (re, re), (im, im), (-im, -im) per entry
              for (int k = 0; k < 4; ++k) {
                const cd e = a[size_t(k)];
                push_coef(bp, cd(e.real(), e.real()));
                push_coef(bp, cd(e.imag(), e.imag()));
                push_coef(bp, cd(-e.imag(), -e.imag()));
              }
            } else {
              for (int k = 0; k < 4; ++k) push_coef(bp, a[size_t(k)]);
            }
            break;
          case LK_D1:
            if (bp.dtype == QSVB_C64) {
              const cd p0 = a[0], p1 = a[3];
              if (in.a == 0) {  // lanes of a float2 pair are the two sides of the gate's bit
                for (int rep = 0; rep < 2; ++rep) {
                  push_coef(bp, cd(p0.real(), p1.real()));
                  push_coef(bp, cd(p0.imag(), p1.imag()));
                  push_coef(bp, cd(-p0.imag(), -p1.imag()));
                }
              } else {
                for (const cd& e : {p0, p1}) {
                  push_coef(bp, cd(e.real(), e.real()));
                  push_coef(bp, cd(e.imag(), e.imag()));
                  push_coef(bp, cd(-e.imag(), -e.imag()));
                }
              }
            } else {
              push_coef(bp, a[0]);
              push_coef(bp, a[3]);
            }
            break;
          case LK_CX:
            in.b = uint32_t(regbit[g.p[1]]);
            break;
          case LK_D1T: {
            in.b = g.t[0];
            for (uint32_t v = 0; v < 2; ++v) {  // the D1 block for tile bit v
              const cd p0 = g.swapq ? a[size_t((v) * 5)] : a[size_t((2 * v) * 5)];
              const cd p1 = g.swapq ? a[size_t((v + 2) * 5)] : a[size_t((1 + 2 * v) * 5)];
              if (bp.dtype == QSVB_C64) {
                if (in.a == 0) {
                  for (int rep = 0; rep < 2; ++rep) {
                    push_coef(bp, cd(p0.real(), p1.real()));
                    push_coef(bp, cd(p0.imag(), p1.imag()));
                    push_coef(bp, cd(-p0.imag(), -p1.imag()));
                  }
                } else {
                  for (const cd& e : {p0, p1}) {
                    push_coef(bp, cd(e.real(), e.real()));
                    push_coef(bp, cd(e.imag(), e.imag()));
                    push_coef(bp, cd(-e.imag(), -e.imag()));
                  }
                }
              } else {
                push_coef(bp, p0);
                push_coef(bp, p1);
              }
            }
            break;
          }
          case LK_D1P:
            in.coef = g.t[0];
            (*tph)[g.t[0]].j0 = in.a == 0;
            break;
          case LK_DTP:
            in.a = 0;
            in.coef = g.t[0];
            break;
          case LK_DT: {
            in.a = 0;
            in.b = g.t[0] | (g.t[1] << 8) | (g.nt << 16);
            const size_t d = size_t(1) << g.g->m;
            for (size_t e = 0; e < d; ++e) push_coef(bp, a[e * d + e]);
            break;
          }
          default: {  // LK_2Q / LK_D2: the kernel wants matrix bit 0 on the lower register bit
            const uint32_t ra = uint32_t(regbit[g.p[0]]), rbit = uint32_t(regbit[g.p[1]]);
            const bool swap = ra > rbit;
            in.a = std::min(ra, rbit);
            in.b = std::max(ra, rbit);
            auto perm = [&](int s) { return swap ? (((s & 1) << 1) | ((s >> 1) & 1)) : s; };
            if (g.kind == LK_2Q) {
              for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c) push_coef(bp, a[size_t(perm(r) * 4 + perm(c))]);
            } else {
              for (int r = 0; r < 4; ++r) push_coef(bp, a[size_t(perm(r) * 4 + perm(r))]);
            }
            break;
          }
        }
        bp.prog.push_back(in);
    };
    auto identity = [](const std::vector<cd>& t) {
      for (const cd& z : t)
        if (z != cd(1, 0)) return false;
      return true;
    };
    for (size_t j = 0; j <= ops.size(); ++j) {
      if (!tables[j].empty() && !identity(tables[j])) emit_table(tables[j]);
      if (j == ops.size()) break;
      if (ops[j].g) emit_one(*ops[j].g);
      else if (ops[j].form == 3) emit_group(ops[j]);
      else emit_split(ops[j]);
    }
    bp.phases[phase_idx].ninstr = uint32_t(bp.prog.size() - phase_pc - 1);
  }
}

}  // namespace

// Passes of circuits[0..ncirc) appended to `bp` (circuit numbers, pass, state, probability and
// <Z_0> offsets all counted from zero within `bp`).
struct BatchPart {
  BatchPlan bp;
  std::vector<std::vector<uint32_t>> circuit_passes;
  std::vector<double> cost;
  double bytes = 0, flops = 0;
};

void plan_batch_part(BatchPart& part, const qsvb_circuit* circuits, size_t ncirc) {
  BatchPlan* bp = &part.bp;
  const int dtype = bp->dtype;
  const uint32_t local_bits = bp->local_bits;
  auto& circuit_passes = part.circuit_passes;
  auto& cost = part.cost;
  circuit_passes.assign(ncirc, {});
  cost.assign(ncirc, 0.0);
  const double eb = dtype == QSVB_C128 ? 16.0 : 8.0;
  double& bytes = part.bytes;
  double& flops = part.flops;
  for (size_t ci = 0; ci < ncirc; ++ci) {
    const qsvb_circuit& c = circuits[ci];
    validate_circuit(&c);
    QSVB_REQUIRE(c.n_qubits <= 30, "batched circuits have at most 30 qubits");
    const uint32_t n = c.n_qubits;
    bp->nq.push_back(n);
    const std::vector<HostGate> gates = fuse_single_qubit_runs(c);
    std::vector<uint32_t> kinds(gates.size());
    for (size_t i = 0; i < gates.size(); ++i) kinds[i] = gate_kind(gates[i]);
    const uint32_t L = std::min(n, local_bits);
    const bool single = n <= local_bits;
    const double amps = std::ldexp(1.0, int(n));
    std::vector<char> done(gates.size(), 0);
    size_t first_open = 0;
    uint64_t state_off = 0;
    if (!single) {
      state_off = bp->state_amps;
      bp->state_amps += uint64_t(1) << n;
    }
    bp->prob_off.push_back(bp->prob_total);
    bp->prob_total += uint64_t(1) << n;
    do {
      while (first_open < gates.size() && done[first_open]) ++first_open;
      // local set: all qubits, or bits 0..4 plus the qubits of the first pending gates
      uint64_t S = 0;
      if (single) {
        S = (1ull << n) - 1ull;
      } else {
        S = (1ull << 5) - 1ull;
        for (size_t i = first_open; i < gates.size() && uint32_t(__builtin_popcountll(S)) < L; ++i) {
          if (done[i]) continue;
          uint64_t m = 0;
          for (uint32_t j = 0; j < gates[i].m; ++j) m |= 1ull << gates[i].q[j];
          if (uint32_t(__builtin_popcountll(S | m)) <= L) S |= m;
        }
        for (uint32_t b = 5; b < n && uint32_t(__builtin_popcountll(S)) < L; ++b) S |= 1ull << b;
      }
      PassDev P{};
      P.circuit = uint32_t(ci);
      P.nlocal = uint32_t(__builtin_popcountll(S));
      uint32_t nl = 0, nn = 0;
      int pos[64];
      for (uint32_t b = 0; b < n; ++b) {
        if ((S >> b) & 1) {
          pos[b] = int(nl);
          P.local[nl++] = uint8_t(b);
        } else {
          pos[b] = -1;
          P.nonlocal[nn++] = uint8_t(b);
        }
      }
      P.nnon = nn;
      P.ntiles = 1u << nn;
      P.state_off = state_off;
      P.prob_off = bp->prob_off.back();
      std::vector<LGate> G;
      uint64_t blocked = 0, dblocked = 0;  // qubits of skipped non-diagonal / diagonal gates
      for (size_t i = first_open; i < gates.size(); ++i) {
        if (done[i]) continue;
        uint64_t m = 0;
        for (uint32_t j = 0; j < gates[i].m; ++j) m |= 1ull << gates[i].q[j];
        const bool diag = kinds[i] == LK_D1 || kinds[i] == LK_D2;
        if ((m & ~S) == 0 && (m & blocked) == 0 && (diag || (m & dblocked) == 0)) {
          done[i] = 1;
          const LGate g{kinds[i],
                        {uint32_t(pos[gates[i].q[0]]), gates[i].m == 2 ? uint32_t(pos[gates[i].q[1]]) : 0u},
                        &gates[i]};
          G.push_back(g);
          flops += amps * (g.kind == LK_1Q ? 16.0 : g.kind == LK_2Q ? 32.0 : g.kind == LK_CX ? 0.0 : 6.0);
        } else if (diag) {
          dblocked |= m;
        } else {
          blocked |= m;
        }
      }
      P.prog_off = uint32_t(bp->prog.size());
      P.phase_off = uint32_t(bp->phases.size());
      P.coef_off = uint32_t(bp->coef.size() / 2);
      emit_phases(*bp, G, P.nlocal);
      P.prog_len = uint32_t(bp->prog.size()) - P.prog_off;
      P.nphase = uint32_t(bp->phases.size()) - P.phase_off;
      P.ncoef = uint32_t(bp->coef.size() / 2) - P.coef_off;
      {
        const size_t rsz = dtype == QSVB_C128 ? 8 : 4;
        const size_t co = (P.prog_len * sizeof(Instr) + P.nphase * sizeof(PhaseDev) + 7) & ~size_t(7);
        P.staged = co + size_t(P.ncoef) * 2 * rsz <= kStageBytes ? 1u : 0u;
      }
      P.first = circuit_passes[ci].empty() ? 1u : 0u;
      P.prev = circuit_passes[ci].empty() ? ~0u : circuit_passes[ci].back();
      circuit_passes[ci].push_back(uint32_t(bp->passes.size()));
      bp->passes.push_back(P);
    } while (std::find(done.begin(), done.end(), char(0)) != done.end());
    // the last pass writes probabilities and <Z_0> partials
    PassDev& last = bp->passes[circuit_passes[ci].back()];
    last.last = 1;
    last.zslot = bp->zslots;
    bp->zoff.push_back(bp->zslots);
    bp->zcnt.push_back(last.ntiles);
    bp->zslots += last.ntiles;
    const size_t np = circuit_passes[ci].size();
    bytes += amps * 8.0 + double(np - 1) * 2.0 * amps * eb;
    cost[ci] = double(np) * amps + double(gates.size()) * amps / 16.0;
  }
}

std::unique_ptr<BatchPlan> build_batch(const qsvb_circuit* circuits, size_t ncirc, int dtype, uint32_t local_bits,
                                       uint32_t reg_bits) {
  QSVB_REQUIRE(circuits != nullptr && ncirc > 0, "empty batch");
  QSVB_REQUIRE(ncirc <= (1u << 20), "at most 2^20 circuits per batch");
  QSVB_REQUIRE(dtype == QSVB_C64 || dtype == QSVB_C128, "dtype must be QSVB_C64 or QSVB_C128");
  QSVB_REQUIRE(local_bits >= 7 && local_bits <= uint32_t(kMaxLocal), "local qubits must be 7..14");
  auto bp = std::make_unique<BatchPlan>();
  bp->dtype = dtype;
  bp->local_bits = local_bits;
  bp->rb = reg_bits;
  bp->swz_w = dtype == QSVB_C128 ? 4u : 5u;
  bp->ncirc = uint32_t(ncirc);
  // circuits are planned independently: contiguous chunks on host threads, then concatenated with
  // their offsets shifted (the result does not depend on the number of chunks)
  size_t nthreads = std::max<size_t>(1, std::thread::hardware_concurrency());
  if (const char* e = std::getenv("QSVB_BATCH_PLAN_THREADS")) nthreads = std::max(1, std::atoi(e));
  const size_t nchunks = std::min<size_t>({nthreads, ncirc, 32});
  std::vector<BatchPart> parts(nchunks);
  std::vector<size_t> lo(nchunks + 1);
  for (size_t k = 0; k <= nchunks; ++k) lo[k] = ncirc * k / nchunks;
  for (BatchPart& pt : parts) {
    pt.bp.dtype = dtype;
    pt.bp.local_bits = local_bits;
    pt.bp.rb = reg_bits;
    pt.bp.swz_w = bp->swz_w;
  }
  if (nchunks == 1) {
    plan_batch_part(parts[0], circuits, ncirc);
  } else {
    std::vector<std::future<void>> fut;
    for (size_t k = 0; k < nchunks; ++k)
      fut.push_back(std::async(std::launch::async, plan_batch_part, std::ref(parts[k]), circuits + lo[k],
                               lo[k + 1] - lo[k]));
    for (auto& f : fut) f.get();
  }
  std::vector<std::vector<uint32_t>> circuit_passes;
  std::vector<double> cost;
  circuit_passes.reserve(ncirc);
  cost.reserve(ncirc);
  double bytes = 0, flops = 0;
  for (size_t k = 0; k < nchunks; ++k) {
    BatchPart& pt = parts[k];
    const BatchPlan& q = pt.bp;
    const uint32_t pass_base = uint32_t(bp->passes.size());
    const uint32_t prog_base = uint32_t(bp->prog.size()), phase_base = uint32_t(bp->phases.size());
    const uint32_t coef_base = uint32_t(bp->coef.size() / 2);
    const uint64_t state_base = bp->state_amps, prob_base = bp->prob_total, z_base = bp->zslots;
    for (PassDev P : q.passes) {
      const bool single = q.nq[P.circuit] <= local_bits;  // whole in shared memory: no state block
      P.circuit += uint32_t(lo[k]);
      if (!single) P.state_off += state_base;
      P.prob_off += prob_base;
      P.prog_off += prog_base;
      P.phase_off += phase_base;
      P.coef_off += coef_base;
      if (P.prev != ~0u) P.prev += pass_base;
      if (P.last) P.zslot += z_base;
      bp->passes.push_back(P);
    }
    bp->phases.insert(bp->phases.end(), q.phases.begin(), q.phases.end());
    bp->prog.insert(bp->prog.end(), q.prog.begin(), q.prog.end());
    bp->coef.insert(bp->coef.end(), q.coef.begin(), q.coef.end());
    bp->nq.insert(bp->nq.end(), q.nq.begin(), q.nq.end());
    for (uint64_t v : q.prob_off) bp->prob_off.push_back(v + prob_base);
    for (uint64_t v : q.zoff) bp->zoff.push_back(v + z_base);
    bp->zcnt.insert(bp->zcnt.end(), q.zcnt.begin(), q.zcnt.end());
    bp->state_amps += q.state_amps;
    bp->prob_total += q.prob_total;
    bp->zslots += q.zslots;
    for (auto& v : pt.circuit_passes) {
      for (uint32_t& pi : v) pi += pass_base;
      circuit_passes.push_back(std::move(v));
    }
    cost.insert(cost.end(), pt.cost.begin(), pt.cost.end());
    bytes += pt.bytes;
    flops += pt.flops;
  }
  // work items: level by level, costliest circuits first within a level
  std::vector<uint32_t> order(ncirc);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
  size_t max_passes = 0;
  for (auto& v : circuit_passes) max_passes = std::max(max_passes, v.size());
  for (size_t lvl = 0; lvl < max_passes; ++lvl)
    for (uint32_t ci : order)
      if (lvl < circuit_passes[ci].size()) {
        const uint32_t pi = circuit_passes[ci][lvl];
        for (uint32_t t = 0; t < bp->passes[pi].ntiles; ++t) bp->items.push_back({pi, t});
      }
  QSVB_REQUIRE(bp->items.size() < (1ull << 31), "batch too large");
  bp->stats.n_gates_in = 0;
  for (size_t ci = 0; ci < ncirc; ++ci) bp->stats.n_gates_in += circuits[ci].n_gates;
  bp->stats.n_sweeps = bp->passes.size();
  bp->stats.n_sweeps_by_kind[0] = bp->phases.size();  // register phases
  bp->stats.algorithmic_bytes = bytes;
  bp->stats.full_sweep_bytes = double(bp->prob_total) * 8.0;
  bp->stats.flops = flops;
  return bp;
}

}  // namespace qsvb

// ----------------------------------------------------------------------------- batch object
struct qsvb_batch {
  std::unique_ptr<qsvb::BatchPlan> plan;
  int device = 0;
  void* d_items = nullptr;
  void* d_passes = nullptr;
  void* d_phases = nullptr;
  void* d_prog = nullptr;
  void* d_coef = nullptr;
  void* d_sre = nullptr;
  void* d_sim = nullptr;
  void* d_zcnt = nullptr;
  void* d_zoff = nullptr;
  double* d_probs = nullptr;
  double* d_zpart = nullptr;
  double* d_z0 = nullptr;
  uint32_t* d_done = nullptr;
  uint32_t* d_queue = nullptr;
  long long* d_prof = nullptr;  // per-block cycle counters (QSVB_BATCH_PROFILE)
  long long* d_wait = nullptr;  // dependency-wait budget in clock64 cycles (qsvb_batch_set_wait_budget)
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int grid = 0;
  size_t smem = 0;
  ~qsvb_batch() {
    if (graph) cudaGraphExecDestroy(graph);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    void* ptrs[] = {d_items, d_passes, d_phases, d_prog, d_coef, d_sre, d_sim, d_zcnt, d_zoff,
                    d_probs, d_zpart, d_z0, d_done, d_queue, d_prof, d_wait};
    for (void* p : ptrs)
      if (p) cudaFree(p);
  }
};

namespace qsvb {
namespace {

template <class T> void upload_vec(void** dst, const std::vector<T>& v, cudaStream_t s) {
  QSVB_CK(cudaMalloc(dst, std::max<size_t>(v.size(), 1) * sizeof(T)));
  if (!v.empty()) QSVB_CK(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

template <class R, int RB, int W, int NT> void configure(qsvb_batch* b, qsvb_ctx* c) {
  auto fn = k_batch<R, RB, W, NT>;
  QSVB_CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(b->smem)));
  QSVB_CK(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                               int(cudaSharedmemCarveoutMaxShared)));
  int occ = 0;
  QSVB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, NT, b->smem));
  QSVB_REQUIRE(occ >= 1, "batched kernel does not fit on an SM");
  b->grid = c->num_sms * occ;
}

template <class R, int RB, int W, int NT> void launch(qsvb_batch* b, qsvb_ctx* c, cudaStream_t s) {
  const BatchPlan& bp = *b->plan;
  k_batch<R, RB, W, NT><<<unsigned(b->grid), NT, b->smem, s>>>(
      static_cast<const Item*>(b->d_items), uint32_t(bp.items.size()), static_cast<const PassDev*>(b->d_passes),
      static_cast<const PhaseDev*>(b->d_phases), static_cast<const Instr*>(b->d_prog),
      static_cast<const R*>(b->d_coef), static_cast<R*>(b->d_sre), static_cast<R*>(b->d_sim), b->d_probs,
      b->d_zpart, b->d_done, b->d_queue, c->d_err, bp.local_bits, b->d_prof, 0u, b->d_wait);
}

// The kernel variants: register bits (a group of 2^RB amplitudes per thread) and block size. The
// widest register tile runs 256 threads with up to 255 registers each; one bit less fits 128
// registers and runs 512 threads.
void configure_any(qsvb_batch* b, qsvb_ctx* c, int dtype, uint32_t rb) {
  if (dtype == QSVB_C128) {
    if (rb == 4) configure<double, 4, 4, 256>(b, c);
    else configure<double, 3, 4, 512>(b, c);
  } else {
    if (rb == 5) configure<float, 5, 5, 256>(b, c);
    else configure<float, 4, 5, 512>(b, c);
  }
}

void launch_any(qsvb_batch* b, qsvb_ctx* c, cudaStream_t s, int dtype, uint32_t rb) {
  if (dtype == QSVB_C128) {
    if (rb == 4) launch<double, 4, 4, 256>(b, c, s);
    else launch<double, 3, 4, 512>(b, c, s);
  } else {
    if (rb == 5) launch<float, 5, 5, 256>(b, c, s);
    else launch<float, 4, 5, 512>(b, c, s);
  }
}

}  // namespace

uint32_t batch_max_local_bits(int dtype) { return dtype == QSVB_C128 ? 13u : 14u; }
uint32_t batch_max_register_bits(int dtype) { return dtype == QSVB_C128 ? 4u : 5u; }

qsvb_batch* batch_create(qsvb_ctx* c, const qsvb_circuit* circuits, size_t n, int dtype, uint32_t local_qubits,
                         uint32_t register_qubits) {
  QSVB_REQUIRE(dtype == QSVB_C64 || dtype == QSVB_C128, "dtype must be QSVB_C64 or QSVB_C128");
  const uint32_t cap = batch_max_local_bits(dtype), rcap = batch_max_register_bits(dtype);
  QSVB_REQUIRE(local_qubits <= cap, "local qubits above " + std::to_string(cap) + " do not fit in shared memory");
  QSVB_REQUIRE(register_qubits == 0 || register_qubits == rcap || register_qubits == rcap - 1,
               "register qubits must be " + std::to_string(rcap - 1) + " or " + std::to_string(rcap));
  const uint32_t regb = register_qubits ? register_qubits : rcap;
  auto b = std::make_unique<qsvb_batch>();
  b->plan = build_batch(circuits, n, dtype, local_qubits ? local_qubits : cap, regb);
  const BatchPlan& bp = *b->plan;
  b->device = c->device;
  const bool f64 = dtype == QSVB_C128;
  const size_t rb = f64 ? 8 : 4;
  {
    size_t free_b = 0, total_b = 0;
    QSVB_CK(cudaMemGetInfo(&free_b, &total_b));
    const double need = double(bp.state_amps) * 2.0 * double(rb) + double(bp.prob_total) * 8.0 +
                        double(bp.items.size()) * sizeof(Item) + double(bp.passes.size()) * (sizeof(PassDev) + 4) +
                        double(bp.prog.size()) * sizeof(Instr) + double(bp.coef.size()) * 8.0;
    if (need > double(free_b))
      throw Error(QSVB_E_OOM, "batch needs " + std::to_string(need / 1e9) + " GB of device memory, " +
                                  std::to_string(double(free_b) / 1e9) + " GB free");
  }
  cudaStream_t s = c->stream;
  upload_vec(&b->d_items, bp.items, s);
  upload_vec(&b->d_passes, bp.passes, s);
  upload_vec(&b->d_phases, bp.phases, s);
  upload_vec(&b->d_prog, bp.prog, s);
  if (f64) {
    upload_vec(&b->d_coef, bp.coef, s);
  } else {
    const std::vector<float> cf(bp.coef.begin(), bp.coef.end());
    upload_vec(&b->d_coef, cf, s);
    QSVB_CK(cudaStreamSynchronize(s));
  }
  upload_vec(&b->d_zcnt, bp.zcnt, s);
  upload_vec(&b->d_zoff, bp.zoff, s);
  QSVB_CK(cudaMalloc(&b->d_sre, std::max<uint64_t>(bp.state_amps, 1) * rb));
  QSVB_CK(cudaMalloc(&b->d_sim, std::max<uint64_t>(bp.state_amps, 1) * rb));
  QSVB_CK(cudaMalloc(reinterpret_cast<void**>(&b->d_probs), bp.prob_total * 8));
  QSVB_CK(cudaMalloc(reinterpret_cast<void**>(&b->d_zpart), bp.zslots * 8));
  QSVB_CK(cudaMalloc(reinterpret_cast<void**>(&b->d_z0), size_t(bp.ncirc) * 8));
  QSVB_CK(cudaMalloc(reinterpret_cast<void**>(&b->d_done), bp.passes.size() * 4));
  QSVB_CK(cudaMalloc(reinterpret_cast<void**>(&b->d_queue), 4));
  QSVB_CK(cudaMalloc(reinterpret_cast<void**>(&b->d_wait), sizeof(long long)));
  {
    const long long budget = kSpinBudget;
    QSVB_CK(cudaMemcpyAsync(b->d_wait, &budget, sizeof(budget), cudaMemcpyHostToDevice, s));
  }
  QSVB_CK(cudaStreamSynchronize(s));
  b->smem = ((size_t(2) * rb) << bp.local_bits) + kStageBytes;
  configure_any(b.get(), c, dtype, regb);
  // QSVB_BATCH_PROFILE=1: per-block cycles spent waiting, filling, in gates and writing out,
  // averaged over blocks and printed to stderr after each run
  if (std::getenv("QSVB_BATCH_PROFILE"))
    QSVB_CK(cudaMalloc(reinterpret_cast<void**>(&b->d_prof), 5 * 8 * size_t(b->grid)));
  QSVB_CK(cudaEventCreate(&b->e0));
  QSVB_CK(cudaEventCreate(&b->e1));
  // the per-run device work as one graph: counter resets, the persistent kernel, the <Z_0> sums
  cudaGraph_t g = nullptr;
  QSVB_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaError_t cap_err = cudaMemsetAsync(b->d_done, 0, bp.passes.size() * 4, s);
  if (cap_err == cudaSuccess) cap_err = cudaMemsetAsync(b->d_queue, 0, 4, s);
  if (cap_err == cudaSuccess) {
    launch_any(b.get(), c, s, dtype, regb);
    cap_err = cudaGetLastError();
  }
  if (cap_err == cudaSuccess) {
    k_batch_z0<<<(bp.ncirc + 255) / 256, 256, 0, s>>>(b->d_zpart, static_cast<const uint64_t*>(b->d_zoff),
                                                       static_cast<const uint32_t*>(b->d_zcnt), bp.ncirc, b->d_z0);
    cap_err = cudaGetLastError();
  }
  const cudaError_t end_err = cudaStreamEndCapture(s, &g);
  if (cap_err != cudaSuccess || end_err != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    QSVB_CK(cap_err);
    QSVB_CK(end_err);
  }
  const cudaError_t inst = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  QSVB_CK(inst);
  return b.release();
}

void batch_set_wait_budget(qsvb_ctx* c, qsvb_batch* b, uint64_t cycles) {
  QSVB_REQUIRE(b != nullptr && b->plan, "null batch");
  QSVB_REQUIRE(b->device == c->device, "batch belongs to another device");
  QSVB_REQUIRE(cycles <= (uint64_t(1) << 40), "wait budget must be at most 2^40 cycles");
  const long long v = cycles == 0 ? kSpinBudget : static_cast<long long>(cycles);
  QSVB_CK(cudaMemcpyAsync(b->d_wait, &v, sizeof(v), cudaMemcpyHostToDevice, c->stream));
  QSVB_CK(cudaStreamSynchronize(c->stream));
}

void batch_run(qsvb_ctx* c, qsvb_batch* b, double* z0_out, double* probs_out, const uint64_t* probs_offset,
               qsvb_plan_stats* stats) {
  QSVB_REQUIRE(b != nullptr && b->plan, "null batch");
  QSVB_REQUIRE(b->device == c->device, "batch belongs to another device");
  const BatchPlan& bp = *b->plan;
  cudaStream_t s = c->stream;
  QSVB_CK(cudaEventRecord(b->e0, s));
  QSVB_CK(cudaGraphLaunch(b->graph, s));
  QSVB_CK(cudaEventRecord(b->e1, s));
  if (z0_out) QSVB_CK(cudaMemcpyAsync(z0_out, b->d_z0, size_t(bp.ncirc) * 8, cudaMemcpyDeviceToHost, s));
  QSVB_CK(cudaStreamSynchronize(s));
  int flag = 0;
  QSVB_CK(cudaMemcpy(&flag, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) {
    QSVB_CK(cudaMemset(c->d_err, 0, sizeof(int)));
    if (flag & kErrBounds)
      throw Error(QSVB_E_CUDA, "a device bounds check failed (an index out of its buffer); results are invalid");
    throw Error(QSVB_E_TIMEOUT, "a batched-runner dependency wait ran out of its budget; results are invalid");
  }
  if (probs_out) {
    if (probs_offset) {
      for (size_t i = 0; i < bp.ncirc; ++i)
        QSVB_CK(cudaMemcpyAsync(probs_out + probs_offset[i], b->d_probs + bp.prob_off[i],
                                (size_t(1) << bp.nq[i]) * 8, cudaMemcpyDeviceToHost, s));
      QSVB_CK(cudaStreamSynchronize(s));
    } else {
      d2h_staged(c, probs_out, b->d_probs, bp.prob_total * 8);
    }
  }
  if (b->d_prof) {
    std::vector<long long> h(5 * size_t(b->grid));
    QSVB_CK(cudaMemcpy(h.data(), b->d_prof, h.size() * 8, cudaMemcpyDeviceToHost));
    double avg[5] = {0, 0, 0, 0, 0};
    for (int i = 0; i < b->grid; ++i)
      for (int j = 0; j < 5; ++j) avg[j] += double(h[5 * size_t(i) + size_t(j)]) / b->grid;
    std::fprintf(stderr,
                 "{\"batch_profile\": {\"wait\": %.0f, \"fill\": %.0f, \"gates\": %.0f, \"out\": %.0f, "
                 "\"items_per_block\": %.1f}}\n",
                 avg[0], avg[1], avg[2], avg[3], avg[4]);
  }
  if (stats) {
    float ms = 0;
    QSVB_CK(cudaEventElapsedTime(&ms, b->e0, b->e1));
    *stats = bp.stats;
    stats->predicted_seconds = 0.0;  // the batched runner predicts nothing
    stats->measured_seconds = double(ms) * 1e-3;  // device seconds of the batched graph
  }
}

// Times every tile shape (local qubits 12 up to the shared-memory limit, either register width) on
// this batch, two runs each with the second timed, and returns the fastest.
void batch_autotune(qsvb_ctx* c, const qsvb_circuit* circuits, size_t n, int dtype, uint32_t* best_local,
                    uint32_t* best_reg, double* seconds, size_t cap, size_t* count) {
  const uint32_t hi = batch_max_local_bits(dtype), rhi = batch_max_register_bits(dtype);
  size_t idx = 0;
  double best_t = 1e300;
  *best_local = hi;
  *best_reg = rhi;
  for (uint32_t L = hi - 2; L <= hi; ++L)
    for (uint32_t rb = rhi - 1; rb <= rhi; ++rb, ++idx) {
      std::unique_ptr<qsvb_batch> b(batch_create(c, circuits, n, dtype, L, rb));
      qsvb_plan_stats st{};
      batch_run(c, b.get(), nullptr, nullptr, nullptr, &st);
      batch_run(c, b.get(), nullptr, nullptr, nullptr, &st);
      if (seconds && idx < cap) seconds[idx] = st.measured_seconds;
      if (st.measured_seconds < best_t) {
        best_t = st.measured_seconds;
        *best_local = L;
        *best_reg = rb;
      }
    }
  if (count) *count = idx;
}

}  // namespace qsvb

void run_batch(qsvb_ctx* c, const qsvb_circuit* circuits, size_t n_circuits, int dtype, uint32_t local_qubits,
               uint32_t register_qubits, double* z0_out, double* probs_out, const uint64_t* probs_offset,
               qsvb_plan_stats* stats) {
  std::unique_ptr<qsvb_batch> b(qsvb::batch_create(c, circuits, n_circuits, dtype, local_qubits, register_qubits));
  qsvb::batch_run(c, b.get(), z0_out, probs_out, probs_offset, stats);
}

void free_batch(qsvb_batch* b) { delete b; }

// ----------------------------------------------------------------------------- tile sweeps
// A tile sweep runs one pass of the batched kernel over one state (any n up to 34): the gates of a
// plan segment that act inside the local set S, applied tile by tile in shared memory, each tile
// read and written once. Blocks take tiles i, i + grid, ... (no queue, no dependencies).
namespace qsvb {

uint32_t tile_local_bits(int dtype, uint32_t n) {
  const uint32_t lmax = batch_max_local_bits(dtype) - 2;  // a 32 KB tile: five blocks per SM
  if (n >= lmax + 8) return lmax;  // at least 256 tiles to spread over the SMs
  if (n >= 15) return n - 8;
  return 0;
}

namespace {
uint32_t tile_reg_bits(int dtype) { return dtype == QSVB_C128 ? 3u : 4u; }
size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
constexpr size_t kTileSmemMax = (size_t(2) * 4 << 12) + kTileStageBytes + kTphSlots * kTphSlotR * 8;

template <class R, int RB, int NT, int MINB, int GP>
void launch_tile_variant(const LaunchEnv& e, R* re, R* im, const Sweep& s, const uint8_t* base) {
  constexpr int W = sizeof(R) == 8 ? 4 : 5;
  auto fn = k_batch<R, RB, W, NT, MINB, GP, kTileHi>;
  QSVB_REQUIRE(s.tile_lbits <= 12 && (1u << (s.tile_lbits - uint32_t(W))) <= uint32_t(kTileHi),
               "tile sweep wider than its address tables");
  static std::once_flag once;
  std::call_once(once, [&] {
    QSVB_CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTileSmemMax)));
    QSVB_CK(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 int(cudaSharedmemCarveoutMaxShared)));
  });
  const size_t smem = ((size_t(2) * sizeof(R)) << s.tile_lbits) + kTileStageBytes + kTphSlots * kTphSlotR * sizeof(R);
  int occ = 0;
  QSVB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, NT, smem));
  QSVB_REQUIRE(occ >= 1, "tile kernel does not fit on an SM");
  const uint32_t grid = uint32_t(std::min<uint64_t>(s.tile_ntiles, uint64_t(e.num_sms) * uint64_t(occ)));
  fn<<<grid, NT, smem, e.stream>>>(nullptr, s.tile_ntiles, reinterpret_cast<const PassDev*>(base),
                                   reinterpret_cast<const PhaseDev*>(base + s.tile_off_phase),
                                   reinterpret_cast<const Instr*>(base + s.tile_off_prog),
                                   reinterpret_cast<const R*>(base + s.tile_off_coef), re, im, nullptr, nullptr,
                                   nullptr, nullptr, e.err_flag, s.tile_lbits, nullptr, 1u, nullptr);
  QSVB_CK(cudaGetLastError());
}
}  // namespace

void tile_prepare(Sweep& s, uint32_t n, int dtype) {
  const uint64_t S = s.tile_mask;
  BatchPlan bp;
  bp.dtype = dtype;
  bp.rb = tile_reg_bits(dtype);
  bp.swz_w = dtype == QSVB_C128 ? 4u : 5u;
  PassDev P{};
  P.nlocal = uint32_t(__builtin_popcountll(S));
  QSVB_REQUIRE((S & 31u) == 31u && P.nlocal >= 7 && P.nlocal <= batch_max_local_bits(dtype) - 2 && n <= QSVB_MAX_QUBITS &&
                   (n >= 64 || (S >> n) == 0),
               "tile sweep: the local set must hold qubits 0..4 and 7..12 (11 for complex128) qubits of the state");
  bp.local_bits = P.nlocal;
  int pos[64];
  uint32_t nl = 0, nn = 0;
  for (uint32_t b = 0; b < n; ++b) {
    if ((S >> b) & 1u) {
      pos[b] = int(nl);
      P.local[nl++] = uint8_t(b);
    } else {
      pos[b] = -1;
      P.nonlocal[nn++] = uint8_t(b);
    }
  }
  P.nnon = nn;
  P.ntiles = 1u << nn;
  P.prev = ~0u;
  const double dim = std::ldexp(1.0, int(n));
  std::vector<HostGate> hg(s.tile_gates.size());
  std::vector<LGate> G;
  double flops = 0;
  for (size_t i = 0; i < s.tile_gates.size(); ++i) {
    const Gate& g = s.tile_gates[i];
    QSVB_REQUIRE(g.m >= 1 && g.m <= 2, "tile sweeps take 1- and 2-qubit gates");
    hg[i].m = g.m;
    hg[i].q[0] = g.q[0];
    hg[i].q[1] = g.m == 2 ? g.q[1] : 0u;
    hg[i].a = g.a;
    uint32_t nout = 0;
    for (uint32_t j = 0; j < g.m; ++j) {
      QSVB_REQUIRE(g.q[j] < n, "tile gate qubit out of range");
      nout += pos[g.q[j]] < 0;
    }
    const uint32_t kind = gate_kind(hg[i]);
    // the tile index bit of a qubit outside the local set
    auto tbit = [&](uint32_t q) {
      for (uint32_t j = 0; j < nn; ++j)
        if (P.nonlocal[j] == q) return j;
      return 0u;
    };
    if (nout == 0) {
      G.push_back(LGate{kind, {uint32_t(pos[g.q[0]]), g.m == 2 ? uint32_t(pos[g.q[1]]) : 0u}, &hg[i]});
    } else {
      QSVB_REQUIRE(kind == LK_D1 || kind == LK_D2, "only diagonal gates may reach qubits outside the tile");
      LGate lg{};
      lg.g = &hg[i];
      if (nout == g.m) {  // all qubits outside: a phase fixed per tile
        lg.kind = LK_DT;
        lg.nt = g.m;
        lg.t[0] = tbit(g.q[0]);
        lg.t[1] = g.m == 2 ? tbit(g.q[1]) : 0u;
      } else {  // one qubit inside, one outside
        lg.kind = LK_D1T;
        lg.swapq = pos[g.q[0]] < 0;
        const uint32_t qin = lg.swapq ? g.q[1] : g.q[0], qout = lg.swapq ? g.q[0] : g.q[1];
        lg.p[0] = uint32_t(pos[qin]);
        lg.t[0] = tbit(qout);
      }
      G.push_back(lg);
    }
  }
  // merge diagonal gates into per-tile phase sums: per local qubit, every diagonal (local or
  // coupled to tile bits) up to the next non-diagonal gate on that qubit; and every diagonal whose
  // qubits are all outside the tile (they commute with the whole pass) into one factor in front
  std::vector<TphOp> tph;
  {
    auto unit = [](const cd& z) { return std::abs(std::abs(z) - 1.0) < 1e-12; };
    std::vector<LGate> out;
    int open[32];
    std::fill(open, open + 32, -1);
    int global = -1;
    std::vector<std::map<uint32_t, std::array<double, 2>>> lin;  // per type-1 op: bit -> (d0, d1)
    std::map<std::pair<uint32_t, uint32_t>, double> quad;         // global op: (k, l) -> angle
    for (const LGate& g : G) {
      const std::vector<cd>& a = g.g->a;
      const size_t d = size_t(1) << g.g->m;
      bool all_unit = true;
      for (size_t e = 0; e < d; ++e) all_unit = all_unit && unit(a[e * d + e]);
      const bool room = tph.size() < kTphSlots;
      if ((g.kind == LK_D1 || g.kind == LK_D1T) && all_unit && (open[g.p[0]] >= 0 || room)) {
        const uint32_t p = g.p[0];
        if (open[p] < 0) {
          open[p] = int(tph.size());
          tph.push_back(TphOp{});
          lin.emplace_back();
          LGate agg{};
          agg.kind = LK_D1P;
          agg.p[0] = p;
          agg.g = g.g;
          agg.t[0] = uint32_t(open[p]);
          out.push_back(agg);
        }
        TphOp& op = tph[size_t(open[p])];
        if (g.kind == LK_D1) {
          op.c0 += std::arg(a[0]);
          op.c1 += std::arg(a[3]);
        } else {
          auto e = [&](int b, int v) { return g.swapq ? a[size_t((v + 2 * b) * 5)] : a[size_t((b + 2 * v) * 5)]; };
          op.c0 += std::arg(e(0, 0));
          op.c1 += std::arg(e(1, 0));
          auto& t = lin[size_t(open[p])][g.t[0]];
          t[0] += std::arg(e(0, 1)) - std::arg(e(0, 0));
          t[1] += std::arg(e(1, 1)) - std::arg(e(1, 0));
        }
        continue;
      }
      if (g.kind == LK_DT && all_unit && (global >= 0 || room)) {
        if (global < 0) {
          global = int(tph.size());
          tph.push_back(TphOp{});
          tph.back().type = 2;
          lin.emplace_back();
        }
        TphOp& op = tph[size_t(global)];
        if (g.nt == 1) {
          op.c0 += std::arg(a[0]);
          quad[{g.t[0], g.t[0]}] += std::arg(a[3]) - std::arg(a[0]);
        } else {
          const double d0 = std::arg(a[0]), d1 = std::arg(a[5]), d2 = std::arg(a[10]), d3 = std::arg(a[15]);
          op.c0 += d0;
          quad[{g.t[0], g.t[0]}] += d1 - d0;
          quad[{g.t[1], g.t[1]}] += d2 - d0;
          quad[{std::min(g.t[0], g.t[1]), std::max(g.t[0], g.t[1])}] += d3 - d1 - d2 + d0;
        }
        continue;
      }
      if (!lgate_diag(g)) {
        for (uint32_t j = 0; j < 32; ++j)
          if ((lgate_mask(g) >> j) & 1u) open[j] = -1;
      }
      out.push_back(g);
    }
    for (size_t i = 0; i < tph.size(); ++i) {
      if (tph[i].type == 1) {
        for (auto& kv : lin[i]) tph[i].terms.push_back({double(kv.first), kv.second[0], kv.second[1]});
      } else {
        for (auto& kv : quad) tph[i].terms.push_back({double(kv.first.first), double(kv.first.second), kv.second});
      }
    }
    if (global >= 0) {
      LGate agg{};
      agg.kind = LK_DTP;
      agg.g = G.front().g;
      agg.t[0] = uint32_t(global);
      out.insert(out.begin(), agg);
    }
    G.swap(out);
  }
  emit_phases(bp, G, P.nlocal, &tph);
  // arithmetic per amplitude of the emitted program, in FP32/FP64 operations: general 1-qubit gates
  // 16, split-form ones 8, 2-qubit dense 32, diagonal kinds 6 (one complex multiply), and each
  // register phase kTilePhaseWork for its shared-memory round trip
  constexpr double kTilePhaseWork = 8.0;
  double work = 0;
  for (const Instr& in : bp.prog) {
    switch (in.op) {
      case OP_PHASE: work += kTilePhaseWork; break;
      case OP_1Q: work += 16.0; break;
      case OP_1QR:
      case OP_1QX: work += 8.0; break;
      case OP_2Q: work += 32.0; break;
      case OP_CX: break;
      default: work += 6.0; break;
    }
  }
  flops = dim * work;
  P.prog_len = uint32_t(bp.prog.size());
  P.nphase = uint32_t(bp.phases.size());
  P.ncoef = uint32_t(bp.coef.size() / 2);
  const size_t rsz = dtype == QSVB_C128 ? 8 : 4;
  {
    const size_t co = (P.prog_len * sizeof(Instr) + P.nphase * sizeof(PhaseDev) + 7) & ~size_t(7);
    P.staged = co + size_t(P.ncoef) * 2 * rsz <= kTileStageBytes ? 1u : 0u;
  }
  const size_t off_phase = align16(sizeof(PassDev));
  const size_t off_prog = align16(off_phase + bp.phases.size() * sizeof(PhaseDev));
  const size_t off_coef = align16(off_prog + bp.prog.size() * sizeof(Instr));
  const size_t off_tph = align16(off_coef + bp.coef.size() * rsz);
  std::vector<uint32_t> toffs;
  std::vector<double> tdat;
  // per operation: type, the factors of both sides with no tile bit set, the term count, then per
  // term (tile bit k, tile bit l, factor of side 0, factor of side 1) applied when bits k and l
  // are set, then the register-bit-0 flag
  for (const TphOp& op : tph) {
    toffs.push_back(uint32_t(tdat.size()));
    tdat.push_back(double(op.type));
    tdat.push_back(std::cos(op.c0));
    tdat.push_back(std::sin(op.c0));
    tdat.push_back(std::cos(op.c1));
    tdat.push_back(std::sin(op.c1));
    tdat.push_back(double(op.terms.size()));
    for (const auto& t : op.terms) {
      const bool lin = op.type == 1;
      const double a0 = lin ? t[1] : t[2], a1 = lin ? t[2] : 0.0;
      tdat.push_back(t[0]);
      tdat.push_back(lin ? t[0] : t[1]);
      tdat.push_back(std::cos(a0));
      tdat.push_back(std::sin(a0));
      tdat.push_back(std::cos(a1));
      tdat.push_back(std::sin(a1));
    }
    tdat.push_back(op.j0 ? 1.0 : 0.0);
  }
  const size_t tph_bytes = tph.empty() ? 0 : ((4 * toffs.size() + 7) & ~size_t(7)) + 8 * tdat.size();
  P.tph_n = uint32_t(tph.size());
  P.tph_off = uint32_t(off_tph);
  const size_t total = off_tph + tph_bytes;
  s.tile_blob.assign(total, 0);
  std::memcpy(s.tile_blob.data(), &P, sizeof(P));
  if (!tph.empty()) {
    std::memcpy(s.tile_blob.data() + off_tph, toffs.data(), 4 * toffs.size());
    std::memcpy(s.tile_blob.data() + off_tph + ((4 * toffs.size() + 7) & ~size_t(7)), tdat.data(), 8 * tdat.size());
  }
  if (!bp.phases.empty()) std::memcpy(s.tile_blob.data() + off_phase, bp.phases.data(), bp.phases.size() * sizeof(PhaseDev));
  if (!bp.prog.empty()) std::memcpy(s.tile_blob.data() + off_prog, bp.prog.data(), bp.prog.size() * sizeof(Instr));
  for (size_t i = 0; i < bp.coef.size(); ++i) {
    if (rsz == 8) {
      std::memcpy(s.tile_blob.data() + off_coef + 8 * i, &bp.coef[i], 8);
    } else {
      const float f = float(bp.coef[i]);
      std::memcpy(s.tile_blob.data() + off_coef + 4 * i, &f, 4);
    }
  }
  s.tile_rb = bp.rb;
  s.tile_lbits = P.nlocal;
  s.tile_ntiles = P.ntiles;
  s.tile_off_phase = uint32_t(off_phase);
  s.tile_off_prog = uint32_t(off_prog);
  s.tile_off_coef = uint32_t(off_coef);
  s.tile_flops = flops;
  s.n_gates = s.tile_gates.size();
}

template <class R>
void launch_tile(const LaunchEnv& e, R* re, R* im, uint32_t n, const Sweep& s, const void* dev_blob) {
  QSVB_REQUIRE(dev_blob != nullptr && !s.tile_blob.empty(), "tile sweep without a program");
  QSVB_REQUIRE(n >= s.tile_lbits, "tile sweep larger than the state");
  const uint8_t* base = static_cast<const uint8_t*>(dev_blob);
  // five blocks per SM (some stream their tiles while others compute; the gates' register phases
  // and shared-memory round trips are latency-bound, so warps per SM set the pace): <= 102
  // registers a thread, the 8 KB program stage and 128-entry address tables
  if constexpr (sizeof(R) == 8) launch_tile_variant<double, 3, 128, 5, 1>(e, re, im, s, base);
  else launch_tile_variant<float, 4, 128, 5, 1>(e, re, im, s, base);
}

template void launch_tile<float>(const LaunchEnv&, float*, float*, uint32_t, const Sweep&, const void*);
template void launch_tile<double>(const LaunchEnv&, double*, double*, uint32_t, const Sweep&, const void*);

}  // namespace qsvb
