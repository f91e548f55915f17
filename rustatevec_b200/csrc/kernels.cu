// CUDA-core sweep kernels and FP64 reductions for the B200 statevector engine (sm_100a).
//
// Layout: the state is Structure-of-Arrays, re[2^n] and im[2^n] in HBM, the layout qsv's
// StateVector uses (crates/qsv-core/src/state/mod.rs:25-29) so `download` is a straight copy.
// Every kernel here is HBM-bound except the dense k>=4 sweeps; each moves 16-byte vectors
// (4 x f32 or 2 x f64 amplitudes per component) and walks the state with a grid-stride loop
// sized to a multiple of the SM count.
//
// Index math follows qsv's layout helpers (crates/qsv-core/src/state/layout.rs:22-86):
// insert_zero_bit(s) anchors a pair/block, scatter_bits/gather_bits map a gate sub-index to
// state bits (bit j of the sub-index <-> qubits[j]).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "qsvb_internal.h"

namespace qsvb {

namespace {

constexpr int kThreads = 256;

template <class R> struct VecT;
template <> struct VecT<float> {
  using T = float4;
  static constexpr int N = 4, LOG = 2;
};
template <> struct VecT<double> {
  using T = double2;
  static constexpr int N = 2, LOG = 1;
};

template <class R> __device__ __forceinline__ void vld(const R* p, R (&x)[VecT<R>::N]);
template <> __device__ __forceinline__ void vld<float>(const float* p, float (&x)[4]) {
  float4 v = *reinterpret_cast<const float4*>(p);
  x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
}
template <> __device__ __forceinline__ void vld<double>(const double* p, double (&x)[2]) {
  double2 v = *reinterpret_cast<const double2*>(p);
  x[0] = v.x; x[1] = v.y;
}
template <class R> __device__ __forceinline__ void vst(R* p, const R (&x)[VecT<R>::N]);
template <> __device__ __forceinline__ void vst<float>(float* p, const float (&x)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(x[0], x[1], x[2], x[3]);
}
template <> __device__ __forceinline__ void vst<double>(double* p, const double (&x)[2]) {
  *reinterpret_cast<double2*>(p) = make_double2(x[0], x[1]);
}

// Work enumerator: work item w -> base index. The low `cb` bits of the base are zero (the chunk
// the item covers), zeros are inserted at the sorted `fixed` positions (all >= cb), and
// `set_mask` is OR'd in (control bits pinned to 1). This is insert_zero_bits (layout.rs:70-86)
// applied to chunks instead of single amplitudes.
struct Enum {
  uint32_t nfixed;
  uint32_t fixed[7];
  uint64_t set_mask;
};

__device__ __forceinline__ uint64_t enum_base(uint64_t w, uint32_t cb, const Enum& e) {
  uint64_t x = w << cb;
#pragma unroll
  for (uint32_t j = 0; j < 7; ++j) {
    if (j < e.nfixed) {
      const uint32_t b = e.fixed[j];
      const uint64_t lo = x & ((1ull << b) - 1ull);
      x = ((x - lo) << 1) | lo;
    }
  }
  return x | e.set_mask;
}

template <class R> struct M2 {
  R a[8];  // g00 re, im, g01 re, im, g10 re, im, g11 re, im
};

template <class R>
__device__ __forceinline__ void cmac(R& yr, R& yi, R ar, R ai, R xr, R xi) {
  yr = fma(ar, xr, yr);
  yr = fma(-ai, xi, yr);
  yi = fma(ar, xi, yi);
  yi = fma(ai, xr, yi);
}

template <class R>
__device__ __forceinline__ void apply2(const M2<R>& g, R& r0, R& i0, R& r1, R& i1) {
  R y0r = 0, y0i = 0, y1r = 0, y1i = 0;
  cmac(y0r, y0i, g.a[0], g.a[1], r0, i0);
  cmac(y0r, y0i, g.a[2], g.a[3], r1, i1);
  cmac(y1r, y1i, g.a[4], g.a[5], r0, i0);
  cmac(y1r, y1i, g.a[6], g.a[7], r1, i1);
  r0 = y0r; i0 = y0i; r1 = y1r; i1 = y1i;
}

__device__ __forceinline__ uint64_t gtid() { return blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t gstride() { return (uint64_t)gridDim.x * blockDim.x; }

// ---------------------------------------------------------------------------------------------
// 1-qubit / controlled-1-qubit butterflies (qsv kernels.cu:52-70 computes the same 2x2 update
// per pair with scalar 8-byte accesses; here every access is a coalesced 16-byte vector).
// ---------------------------------------------------------------------------------------------

// Target bit inside one 16-byte vector: pairs are formed in registers.
template <class R, int T>
__global__ void __launch_bounds__(kThreads) k_pair_invec(R* __restrict__ re, R* __restrict__ im,
                                                         uint64_t nwork, Enum en, uint32_t ctrl_low,
                                                         M2<R> g) {
  // the target bit T is a template parameter: with a run-time bit the partner index e | 1 << t
  // indexes the register array dynamically, which puts it in local memory
  constexpr int N = VecT<R>::N, LOG = VecT<R>::LOG;
  static_assert(T < LOG, "in-vector target");
  constexpr uint32_t t = T;
  for (uint64_t w = gtid(); w < nwork; w += gstride()) {
    const uint64_t b = enum_base(w, LOG, en);
    R xr[N], xi[N];
    vld(re + b, xr);
    vld(im + b, xi);
#pragma unroll
    for (int e = 0; e < N; ++e) {
      if (((e >> t) & 1) == 0 && (uint32_t(e) & ctrl_low) == ctrl_low) {
        const int f = e | (1 << t);
        apply2(g, xr[e], xi[e], xr[f], xi[f]);
      }
    }
    vst(re + b, xr);
    vst(im + b, xi);
  }
}

// Target bit within one warp's 32 contiguous vectors: each lane loads its own vector (the warp
// reads 512 contiguous bytes per component) and fetches its partner with a warp shuffle, so
// every HBM sector is read and written exactly once.
template <class R>
__global__ void __launch_bounds__(kThreads) k_pair_shfl(R* __restrict__ re, R* __restrict__ im,
                                                        uint64_t nwork, Enum en, uint32_t t,
                                                        uint32_t ctrl_low, M2<R> g) {
  constexpr int N = VecT<R>::N, LOG = VecT<R>::LOG;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lanemask = 1u << (t - LOG);
  const bool upper = (lane & lanemask) != 0;
  const uint64_t nwarps = gstride() >> 5;
  for (uint64_t w = gtid() >> 5; w < nwork; w += nwarps) {
    const uint64_t b = enum_base(w, LOG + 5, en) + uint64_t(lane) * N;
    R xr[N], xi[N];
    vld(re + b, xr);
    vld(im + b, xi);
#pragma unroll
    for (int e = 0; e < N; ++e) {
      const R pr = __shfl_xor_sync(0xffffffffu, xr[e], lanemask);
      const R pi = __shfl_xor_sync(0xffffffffu, xi[e], lanemask);
      if (((lane * N + e) & ctrl_low) == ctrl_low) {
        R yr = 0, yi = 0;
        if (upper) {  // this lane holds |1>: y = g10 x0 + g11 x1
          cmac(yr, yi, g.a[4], g.a[5], pr, pi);
          cmac(yr, yi, g.a[6], g.a[7], xr[e], xi[e]);
        } else {      // y = g00 x0 + g01 x1
          cmac(yr, yi, g.a[0], g.a[1], xr[e], xi[e]);
          cmac(yr, yi, g.a[2], g.a[3], pr, pi);
        }
        xr[e] = yr;
        xi[e] = yi;
      }
    }
    vst(re + b, xr);
    vst(im + b, xi);
  }
}

// Target bit above one warp's span: each thread owns a vector pair 2^t apart; a warp's 32 lanes
// still read 512 contiguous bytes per access.
template <class R>
__global__ void __launch_bounds__(kThreads) k_pair_strided(R* __restrict__ re, R* __restrict__ im,
                                                           uint64_t nwork, Enum en, uint32_t t,
                                                           uint32_t ctrl_low, M2<R> g) {
  constexpr int N = VecT<R>::N, LOG = VecT<R>::LOG;
  const uint64_t half = 1ull << t;
  for (uint64_t w = gtid(); w < nwork; w += gstride()) {
    const uint64_t b = enum_base(w, LOG, en);
    R r0[N], i0[N], r1[N], i1[N];
    vld(re + b, r0);
    vld(im + b, i0);
    vld(re + b + half, r1);
    vld(im + b + half, i1);
#pragma unroll
    for (int e = 0; e < N; ++e)
      if ((uint32_t(e) & ctrl_low) == ctrl_low) apply2(g, r0[e], i0[e], r1[e], i1[e]);
    vst(re + b, r0);
    vst(im + b, i0);
    vst(re + b + half, r1);
    vst(im + b + half, i1);
  }
}

// Scalar fallback for tiny states: one pair per thread (fixed = sorted {t} U controls).
template <class R>
__global__ void k_pair_scalar(R* __restrict__ re, R* __restrict__ im, uint64_t nwork, Enum en,
                              uint32_t t, M2<R> g) {
  for (uint64_t w = gtid(); w < nwork; w += gstride()) {
    const uint64_t a0 = enum_base(w, 0, en), a1 = a0 | (1ull << t);
    R r0 = re[a0], i0 = im[a0], r1 = re[a1], i1 = im[a1];
    apply2(g, r0, i0, r1, i1);
    re[a0] = r0; im[a0] = i0; re[a1] = r1; im[a1] = i1;
  }
}

// ---------------------------------------------------------------------------------------------
// Diagonal sweep: psi_i *= d[gather_bits(i, qs)] (qsv kernels.cu:73-85 / cpu.rs:100-146). The
// table lives in shared memory; qubits whose 0-half is the identity are pinned to 1 by the
// enumerator so those amplitudes are never touched (CZ / CPHASE touch a quarter of the state).
// ---------------------------------------------------------------------------------------------
template <class R> struct DiagP {
  uint32_t m;
  uint32_t q[6];
  R d[128];  // interleaved (re, im), 2^m entries
};

template <class R>
__global__ void __launch_bounds__(kThreads) k_diag(R* __restrict__ re, R* __restrict__ im,
                                                   uint64_t nwork, Enum en, DiagP<R> p) {
  constexpr int N = VecT<R>::N, LOG = VecT<R>::LOG;
  __shared__ R tab[128];
  for (int i = threadIdx.x; i < (2 << p.m); i += blockDim.x) tab[i] = p.d[i];
  __syncthreads();
  uint32_t lowsub[N];
#pragma unroll
  for (int e = 0; e < N; ++e) {
    uint32_t s = 0;
    for (uint32_t j = 0; j < p.m; ++j)
      if (p.q[j] < uint32_t(LOG)) s |= ((uint32_t(e) >> p.q[j]) & 1u) << j;
    lowsub[e] = s;
  }
  for (uint64_t w = gtid(); w < nwork; w += gstride()) {
    const uint64_t b = enum_base(w, LOG, en);
    uint32_t shi = 0;
    for (uint32_t j = 0; j < p.m; ++j) shi |= uint32_t((b >> p.q[j]) & 1ull) << j;
    R xr[N], xi[N];
    vld(re + b, xr);
    vld(im + b, xi);
#pragma unroll
    for (int e = 0; e < N; ++e) {
      const uint32_t s = shi | lowsub[e];
      const R dr = tab[2 * s], di = tab[2 * s + 1];
      const R a = xr[e], c = xi[e];
      xr[e] = fma(dr, a, -di * c);
      xi[e] = fma(dr, c, di * a);
    }
    vst(re + b, xr);
    vst(im + b, xi);
  }
}

template <class R>
__global__ void k_diag_scalar(R* __restrict__ re, R* __restrict__ im, uint64_t dim, DiagP<R> p) {
  for (uint64_t i = gtid(); i < dim; i += gstride()) {
    uint32_t s = 0;
    for (uint32_t j = 0; j < p.m; ++j) s |= uint32_t((i >> p.q[j]) & 1ull) << j;
    const R dr = p.d[2 * s], di = p.d[2 * s + 1];
    const R a = re[i], c = im[i];
    re[i] = fma(dr, a, -di * c);
    im[i] = fma(dr, c, di * a);
  }
}

// ---------------------------------------------------------------------------------------------
// Phase-polynomial sweep: psi_i *= exp(i * sum_t ang_t[gather_bits(i, q_t)]) over many <= 2-qubit
// diagonal terms (a whole QAOA cost layer of RZZ gates in one pass). The phase is summed and
// evaluated in FP64 for both precisions.
// ---------------------------------------------------------------------------------------------
struct PhaseTermDev {
  uint32_t q0, q1;  // q1 == 64 for a 1-qubit term
  double ang[4];
};

template <class R>
__global__ void __launch_bounds__(kThreads) k_phase(R* __restrict__ re, R* __restrict__ im,
                                                    uint64_t dim, const PhaseTermDev* __restrict__ terms,
                                                    uint32_t nterms) {
  extern __shared__ char smem_raw[];
  PhaseTermDev* st = reinterpret_cast<PhaseTermDev*>(smem_raw);
  for (uint32_t i = threadIdx.x; i < nterms; i += blockDim.x) st[i] = terms[i];
  __syncthreads();
  constexpr int N = VecT<R>::N;
  const uint64_t nvec = dim / N;
  for (uint64_t w = gtid(); w < nvec; w += gstride()) {
    const uint64_t b = w * N;
    R xr[N], xi[N];
    vld(re + b, xr);
    vld(im + b, xi);
#pragma unroll
    for (int e = 0; e < N; ++e) {
      const uint64_t i = b + e;
      double th = 0.0;
      for (uint32_t k = 0; k < nterms; ++k) {
        const PhaseTermDev& T = st[k];
        const uint32_t s = uint32_t((i >> T.q0) & 1ull) | (T.q1 < 64 ? uint32_t((i >> T.q1) & 1ull) << 1 : 0u);
        th += T.ang[s];
      }
      double sn, cs;
      sincos(th, &sn, &cs);
      const double a = double(xr[e]), c = double(xi[e]);
      xr[e] = R(cs * a - sn * c);
      xi[e] = R(cs * c + sn * a);
    }
    vst(re + b, xr);
    vst(im + b, xi);
  }
}

// Phase polynomial in Ising form for states of >= 12 qubits. Any product of <= 2-qubit diagonal
// phases is exp(i theta(x)) with theta = C + sum_q h_q z_q + sum_(a<b) J_ab z_a z_b, z_q = 1 - 2 x_q.
// A CTA walks chunks of 4096 consecutive amplitudes. The edge terms inside the low 12 bits are
// tabulated once per CTA; per chunk, the high bits are constant, so the high-high terms fold into one
// scalar and the high-low edges into the linear coefficients of the low bits, kept as two 64-entry
// tables. All three tables hold unit complex factors exp(i angle) (the chunk scalar folded into the
// first 64-entry one), so an amplitude's factor is a product of three shared loads: two complex
// multiplies in FP64 instead of one sincos per amplitude. The low-bit table is 64 KB of dynamic
// shared memory.
constexpr int kIsingMaxEdges = 160;
constexpr int kIsingChunkBits = 12;
struct IsingP {
  double c0;
  double h[64];
  double J[kIsingMaxEdges];
  uint8_t ea[kIsingMaxEdges], eb[kIsingMaxEdges];  // ea < eb
  uint32_t nedges;
};

__device__ __forceinline__ double zsign(uint64_t x, uint32_t q) { return 1.0 - 2.0 * double((x >> q) & 1ull); }

template <class R>
__global__ void __launch_bounds__(kThreads) k_ising(R* __restrict__ re, R* __restrict__ im, uint64_t nchunks,
                                                    IsingP p) {
  constexpr int CB = kIsingChunkBits, CH = 1 << CB, N = VecT<R>::N;
  extern __shared__ double2 tll[];  // CH entries: (cos, sin) of the low-bit edge phases
  __shared__ double2 l1[64], l2[64];
  __shared__ double hp[CB];
  __shared__ double thh;
  const int tid = threadIdx.x;
  for (int l = tid; l < CH; l += kThreads) {
    double s = 0.0;
    for (uint32_t e = 0; e < p.nedges; ++e)
      if (p.eb[e] < CB) s += p.J[e] * zsign(uint64_t(l), p.ea[e]) * zsign(uint64_t(l), p.eb[e]);
    double sn, cs;
    sincos(s, &sn, &cs);
    tll[l] = make_double2(cs, sn);
  }
  for (uint64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const uint64_t base = ch << CB;
    __syncthreads();  // the previous chunk is done with l1 / l2 / thh (and tll is built)
    if (tid < CB) {
      double v = p.h[tid];
      for (uint32_t e = 0; e < p.nedges; ++e)
        if (p.ea[e] == uint32_t(tid) && p.eb[e] >= CB) v += p.J[e] * zsign(base, p.eb[e]);
      hp[tid] = v;
    } else if (tid == 32) {
      double v = p.c0;
      for (uint32_t q = CB; q < 64; ++q)
        if (p.h[q] != 0.0) v += p.h[q] * zsign(base, q);
      for (uint32_t e = 0; e < p.nedges; ++e)
        if (p.ea[e] >= CB) v += p.J[e] * zsign(base, p.ea[e]) * zsign(base, p.eb[e]);
      thh = v;
    }
    __syncthreads();
    if (tid < 64) {
      double v = thh;
      for (int q = 0; q < 6; ++q) v += hp[q] * zsign(uint64_t(tid), q);
      double sn, cs;
      sincos(v, &sn, &cs);
      l1[tid] = make_double2(cs, sn);
    } else if (tid < 128) {
      double v = 0.0;
      for (int q = 0; q < 6; ++q) v += hp[6 + q] * zsign(uint64_t(tid - 64), q);
      double sn, cs;
      sincos(v, &sn, &cs);
      l2[tid - 64] = make_double2(cs, sn);
    }
    __syncthreads();
    for (int v = tid; v < CH / N; v += kThreads) {
      const uint32_t l = uint32_t(v * N);
      R xr[N], xi[N];
      vld(re + base + l, xr);
      vld(im + base + l, xi);
#pragma unroll
      for (int e = 0; e < N; ++e) {
        const uint32_t x = l + e;
        const double2 f0 = tll[x], f1 = l1[x & 63u], f2 = l2[x >> 6];
        const double ur = f0.x * f1.x - f0.y * f1.y, ui = f0.x * f1.y + f0.y * f1.x;
        const double cs = ur * f2.x - ui * f2.y, sn = ur * f2.y + ui * f2.x;
        const double a = double(xr[e]), c = double(xi[e]);
        xr[e] = R(cs * a - sn * c);
        xi[e] = R(cs * c + sn * a);
      }
      vst(re + base + l, xr);
      vst(im + base + l, xi);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Dense k-qubit sweep on CUDA cores (qsv kernels.cu:91-120 gathers one 2^m block per thread into
// local arrays; here a CTA gathers a tile of 2^K rows x NC columns into shared memory, where the
// columns are the NCB lowest non-gate bits, so every global access is a contiguous run of at least
// NC amplitudes; the tile is then a small complex GEMM Y = U X with U staged in shared memory).
// ---------------------------------------------------------------------------------------------
struct DenseP {
  uint32_t hibits[6];   // tile bits above NCB-1 (ascending), K of them
  uint64_t hioff[64];   // address offset of the high tile bits
  uint32_t dsthi[64];   // shared-memory offset of the high tile bits
  uint32_t dstlo[256];  // shared-memory offset of the low NCB address bits
  uint32_t vecstore;    // 1 when the low LOG address bits are column bits
};

// cp.async copies global -> shared (16 bytes cached in L2 only, or one 4- / 8-byte element).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
template <class R> __device__ __forceinline__ void cp_async_elem(R* dst, const R* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src), "n"(int(sizeof(R)))
               : "memory");
}

// DB: two tile buffers, the gather of tile i + grid (cp.async) in flight while tile i is
// multiplied and written back; otherwise one buffer, gathered with vector loads.
template <class R, int K, int NCB, bool DB>
__global__ void __launch_bounds__(kThreads) k_dense(R* __restrict__ re, R* __restrict__ im,
                                                    uint64_t ntiles, const R* __restrict__ ut,
                                                    DenseP p) {
  constexpr int M = 1 << K, NC = 1 << NCB, N = VecT<R>::N;
  constexpr int RG = kThreads / NC;  // row groups
  constexpr int RPT = M / RG;        // rows per thread
  constexpr int NB = DB ? 2 : 1;     // tile buffers
  static_assert(RG * NC == kThreads && RPT * RG == M, "tile shape");
  extern __shared__ __align__(16) char smem_raw[];
  R* xbuf = reinterpret_cast<R*>(smem_raw);  // buffer b: re [M * NC], im [M * NC]
  R* us = xbuf + NB * 2 * M * NC;            // [s][r] complex interleaved
  uint32_t* dlo = reinterpret_cast<uint32_t*>(us + 2 * M * M);
  uint32_t* dhi = dlo + NC;
  uint64_t* hio = reinterpret_cast<uint64_t*>(dhi + M);  // 8-byte aligned: NC + M is even
  for (int i = threadIdx.x; i < 2 * M * M; i += kThreads) us[i] = ut[i];
  for (int i = threadIdx.x; i < NC; i += kThreads) dlo[i] = p.dstlo[i];
  for (int i = threadIdx.x; i < M; i += kThreads) {
    dhi[i] = p.dsthi[i];
    hio[i] = p.hioff[i];
  }
  const int col = threadIdx.x % NC, rg = threadIdx.x / NC;
  const bool vs = p.vecstore != 0;
  auto tile_base = [&](uint64_t tile) {
    uint64_t base = tile << NCB;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const uint32_t b = p.hibits[j];
      const uint64_t lo = base & ((1ull << b) - 1ull);
      base = ((base - lo) << 1) | lo;
    }
    return base;
  };
  // the tile's gather into buffer b: contiguous runs of >= NC amplitudes, scattered into the
  // (row, column) tile layout
  auto gather = [&](uint64_t base, int b) {
    R* xr = xbuf + b * 2 * M * NC;
    R* xi = xr + M * NC;
    for (int v = threadIdx.x; v < M * NC / N; v += kThreads) {
      const int t = v * N, tlo = t & (NC - 1), thi = t >> NCB;
      const uint64_t a = base + hio[thi] + uint64_t(tlo);
      if constexpr (DB) {
        if (vs) {
          const uint32_t d = dlo[tlo] + dhi[thi];
          cp_async16(xr + d, re + a);
          cp_async16(xi + d, im + a);
        } else {
#pragma unroll
          for (int e = 0; e < N; ++e) {
            const uint32_t d = dlo[tlo + e] + dhi[thi];
            cp_async_elem(xr + d, re + a + e);
            cp_async_elem(xi + d, im + a + e);
          }
        }
      } else {
        R vr[N], vi[N];
        vld(re + a, vr);
        vld(im + a, vi);
        if (vs) {
          const uint32_t d = dlo[tlo] + dhi[thi];
          vst(xr + d, vr);
          vst(xi + d, vi);
        } else {
#pragma unroll
          for (int e = 0; e < N; ++e) {
            const uint32_t d = dlo[tlo + e] + dhi[thi];
            xr[d] = vr[e];
            xi[d] = vi[e];
          }
        }
      }
    }
  };
  __syncthreads();  // tables ready
  if constexpr (DB) {
    if (blockIdx.x < ntiles) gather(tile_base(blockIdx.x), 0);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  int cur = 0;
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, cur ^= NB - 1) {
    const uint64_t base = tile_base(tile);
    if constexpr (DB) {
      // the next tile's gather goes into the other buffer (its last reads ended at the barrier
      // closing the previous iteration); then wait for this tile's group only
      const uint64_t nxt = tile + gridDim.x;
      if (nxt < ntiles) gather(tile_base(nxt), cur ^ 1);
      asm volatile("cp.async.commit_group;" ::: "memory");
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      gather(base, 0);
    }
    __syncthreads();
    R* xr = xbuf + cur * 2 * M * NC;
    R* xi = xr + M * NC;
    R ar[RPT], ai[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) ar[r] = ai[r] = R(0);
#pragma unroll 4
    for (int s = 0; s < M; ++s) {
      const R vr = xr[s * NC + col], vi = xi[s * NC + col];
      const R* u = us + 2 * (s * M + rg * RPT);
#pragma unroll
      for (int r = 0; r < RPT; ++r) cmac(ar[r], ai[r], u[2 * r], u[2 * r + 1], vr, vi);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      xr[(rg * RPT + r) * NC + col] = ar[r];
      xi[(rg * RPT + r) * NC + col] = ai[r];
    }
    __syncthreads();
    for (int v = threadIdx.x; v < M * NC / N; v += kThreads) {
      const int t = v * N, tlo = t & (NC - 1), thi = t >> NCB;
      const uint64_t a = base + hio[thi] + uint64_t(tlo);
      R vr[N], vi[N];
      if (vs) {
        const uint32_t d = dlo[tlo] + dhi[thi];
        vld(xr + d, vr);
        vld(xi + d, vi);
      } else {
#pragma unroll
        for (int e = 0; e < N; ++e) {
          const uint32_t d = dlo[tlo + e] + dhi[thi];
          vr[e] = xr[d];
          vi[e] = xi[d];
        }
      }
      vst(re + a, vr);
      vst(im + a, vi);
    }
    __syncthreads();  // this buffer's reads are done before a later gather reuses it
  }
  if constexpr (DB) asm volatile("cp.async.wait_all;" ::: "memory");
}

// Small-state fallback: one 2^K block per thread (gather, matvec, scatter).
template <class R, int K>
__global__ void k_dense_small(R* __restrict__ re, R* __restrict__ im, uint64_t nblocks,
                              const R* __restrict__ ut, Enum en, uint32_t q0, uint32_t q1,
                              uint32_t q2, uint32_t q3, uint32_t q4, uint32_t q5) {
  constexpr int M = 1 << K;
  const R* __restrict__ us = ut;  // small states only: the matrix stays in L1/L2
  const uint32_t qs[6] = {q0, q1, q2, q3, q4, q5};
  for (uint64_t w = gtid(); w < nblocks; w += gstride()) {
    const uint64_t base = enum_base(w, 0, en);
    R xr[M], xi[M];
#pragma unroll
    for (int s = 0; s < M; ++s) {
      uint64_t idx = base;
#pragma unroll
      for (int j = 0; j < K; ++j) idx |= uint64_t((s >> j) & 1) << qs[j];
      xr[s] = re[idx];
      xi[s] = im[idx];
    }
#pragma unroll 1
    for (int r = 0; r < M; ++r) {
      R yr = 0, yi = 0;
#pragma unroll
      for (int s = 0; s < M; ++s) cmac(yr, yi, us[2 * (s * M + r)], us[2 * (s * M + r) + 1], xr[s], xi[s]);
      uint64_t idx = base;
#pragma unroll
      for (int j = 0; j < K; ++j) idx |= uint64_t((r >> j) & 1) << qs[j];
      re[idx] = yr;
      im[idx] = yi;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// State preparation
// ---------------------------------------------------------------------------------------------
template <class R> __global__ void k_set_one(R* re, uint64_t i) { re[i] = R(1); }

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Counter-based complex Gaussian: two SplitMix64 outputs of (seed, index) -> Box-Muller.
template <class R>
__global__ void k_gaussian(R* __restrict__ re, R* __restrict__ im, uint64_t dim, uint64_t seed) {
  const uint64_t G = 0x9E3779B97F4A7C15ull;
  for (uint64_t i = gtid(); i < dim; i += gstride()) {
    const uint64_t h1 = mix64(seed + (2 * i + 1) * G), h2 = mix64(seed + (2 * i + 2) * G);
    const double u1 = double((h1 >> 11) + 1) * 0x1.0p-53;  // (0, 1]
    const double u2 = double(h2 >> 11) * 0x1.0p-53;        // [0, 1)
    const double r = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    re[i] = R(r * cs);
    im[i] = R(r * sn);
  }
}

template <class R>
__global__ void k_scale(R* __restrict__ re, R* __restrict__ im, uint64_t dim, const double* d_norm) {
  const double inv = 1.0 / sqrt(d_norm[0]);
  for (uint64_t i = gtid(); i < dim; i += gstride()) {
    re[i] = R(double(re[i]) * inv);
    im[i] = R(double(im[i]) * inv);
  }
}

// ---------------------------------------------------------------------------------------------
// FP64 reductions (norm, <Z_mask>, <a|b>): grid-stride partial sums per CTA, then one CTA sums
// the partials in a fixed order (deterministic, no atomics).
// ---------------------------------------------------------------------------------------------
constexpr int kReduceBlocksPerSM = 4;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void block_sum2(double& a, double& b) {
  __shared__ double sa[32], sb[32];
  a = warp_sum(a);
  b = warp_sum(b);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sa[wid] = a;
    sb[wid] = b;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    a = lane < nw ? sa[lane] : 0.0;
    b = lane < nw ? sb[lane] : 0.0;
    a = warp_sum(a);
    b = warp_sum(b);
  }
}

template <class R>
__global__ void __launch_bounds__(kThreads) k_reduce(int op, const R* __restrict__ re, const R* __restrict__ im,
                                                     const R* __restrict__ re2, const R* __restrict__ im2,
                                                     uint64_t dim, uint64_t mask, double* partials) {
  constexpr int N = VecT<R>::N;
  double a = 0.0, b = 0.0;
  if (dim % N == 0) {
    const uint64_t nvec = dim / N;
    for (uint64_t w = gtid(); w < nvec; w += gstride()) {
      R xr[N], xi[N];
      vld(re + w * N, xr);
      vld(im + w * N, xi);
      if (op == RED_INNER) {
        R yr[N], yi[N];
        vld(re2 + w * N, yr);
        vld(im2 + w * N, yi);
#pragma unroll
        for (int e = 0; e < N; ++e) {  // conj(x) * y
          a += double(xr[e]) * double(yr[e]) + double(xi[e]) * double(yi[e]);
          b += double(xr[e]) * double(yi[e]) - double(xi[e]) * double(yr[e]);
        }
      } else {
#pragma unroll
        for (int e = 0; e < N; ++e) {
          const double p = double(xr[e]) * double(xr[e]) + double(xi[e]) * double(xi[e]);
          if (op == RED_EXPZ && (__popcll((w * N + e) & mask) & 1)) a -= p;
          else a += p;
        }
      }
    }
  } else {
    for (uint64_t i = gtid(); i < dim; i += gstride()) {
      const double xr = re[i], xi = im[i];
      if (op == RED_INNER) {
        a += xr * double(re2[i]) + xi * double(im2[i]);
        b += xr * double(im2[i]) - xi * double(re2[i]);
      } else {
        const double p = xr * xr + xi * xi;
        if (op == RED_EXPZ && (__popcll(i & mask) & 1)) a -= p;
        else a += p;
      }
    }
  }
  block_sum2(a, b);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = a;
    partials[2 * blockIdx.x + 1] = b;
  }
}

template <class R> __device__ __forceinline__ void load4(const R* p, R (&x)[4]) {
  if constexpr (sizeof(R) == 4) {
    vld(p, x);
  } else {
    R a[2], b[2];
    vld(p, a);
    vld(p + 2, b);
    x[0] = a[0]; x[1] = a[1]; x[2] = b[0]; x[3] = b[1];
  }
}

// <a|b> across precisions (complex64 state vs its FP64 twin), FP64 accumulation.
template <class RA, class RB>
__global__ void __launch_bounds__(kThreads) k_inner_mixed(const RA* __restrict__ are, const RA* __restrict__ aim,
                                                          const RB* __restrict__ bre, const RB* __restrict__ bim,
                                                          uint64_t dim, double* partials) {
  double a = 0.0, b = 0.0;
  if (dim % 4 == 0) {
    for (uint64_t w = gtid(); w < dim / 4; w += gstride()) {
      RA xr[4], xi[4];
      RB yr[4], yi[4];
      load4(are + 4 * w, xr);
      load4(aim + 4 * w, xi);
      load4(bre + 4 * w, yr);
      load4(bim + 4 * w, yi);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        a += double(xr[e]) * double(yr[e]) + double(xi[e]) * double(yi[e]);
        b += double(xr[e]) * double(yi[e]) - double(xi[e]) * double(yr[e]);
      }
    }
  } else {
    for (uint64_t i = gtid(); i < dim; i += gstride()) {
      a += double(are[i]) * double(bre[i]) + double(aim[i]) * double(bim[i]);
      b += double(are[i]) * double(bim[i]) - double(aim[i]) * double(bre[i]);
    }
  }
  block_sum2(a, b);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = a;
    partials[2 * blockIdx.x + 1] = b;
  }
}

__global__ void k_finalize(const double* partials, int nparts, double* out) {
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    a += partials[2 * i];
    b += partials[2 * i + 1];
  }
  block_sum2(a, b);
  if (threadIdx.x == 0) {
    out[0] = a;
    out[1] = b;
  }
}

template <class R>
__global__ void k_probs(const R* __restrict__ re, const R* __restrict__ im, uint64_t off, uint64_t count,
                        void* out, int out_f64) {
  for (uint64_t i = gtid(); i < count; i += gstride()) {
    const double xr = re[off + i], xi = im[off + i];
    const double p = xr * xr + xi * xi;
    if (out_f64) static_cast<double*>(out)[i] = p;
    else static_cast<float*>(out)[i] = float(p);
  }
}

// ---------------------------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------------------------
inline unsigned grid_for(uint64_t items, int per_block, int num_sms, int blocks_per_sm = 8) {
  const uint64_t need = (items + per_block - 1) / per_block;
  const uint64_t cap = uint64_t(num_sms) * blocks_per_sm;
  return unsigned(std::max<uint64_t>(1, std::min(need, cap)));
}

inline void check_launch() { QSVB_CK(cudaGetLastError()); }

template <class R> M2<R> to_m2(const std::vector<cd>& u) {
  M2<R> g;
  for (int i = 0; i < 4; ++i) {
    g.a[2 * i] = R(u[i].real());
    g.a[2 * i + 1] = R(u[i].imag());
  }
  return g;
}

Enum make_enum(std::vector<uint32_t> fixed, uint64_t set_mask) {
  Enum e{};
  std::sort(fixed.begin(), fixed.end());
  QSVB_REQUIRE(fixed.size() <= 7, "too many fixed bits");
  e.nfixed = uint32_t(fixed.size());
  for (size_t i = 0; i < fixed.size(); ++i) e.fixed[i] = fixed[i];
  e.set_mask = set_mask;
  return e;
}

template <class R>
void launch_pair(const LaunchEnv& env, R* re, R* im, uint32_t n, uint32_t t, const uint32_t* ctrl,
                 uint32_t nctrl, const std::vector<cd>& u) {
  constexpr uint32_t LOG = VecT<R>::LOG;
  const M2<R> g = to_m2<R>(u);
  uint64_t cmask = 0;
  for (uint32_t i = 0; i < nctrl; ++i) cmask |= 1ull << ctrl[i];
  auto split = [&](uint32_t cb, std::vector<uint32_t>& fixed, uint32_t& low) {
    low = 0;
    uint64_t set = 0;
    for (uint32_t i = 0; i < nctrl; ++i) {
      if (ctrl[i] >= cb) {
        fixed.push_back(ctrl[i]);
        set |= 1ull << ctrl[i];
      } else {
        low |= 1u << ctrl[i];
      }
    }
    return set;
  };
  const uint32_t nfix_ctrl_hi_max = nctrl;
  if (n >= 12 && n >= LOG + 6 + nfix_ctrl_hi_max) {
    std::vector<uint32_t> fixed;
    uint32_t low;
    if (t < LOG) {
      const uint64_t set = split(LOG, fixed, low);
      const uint64_t nwork = 1ull << (n - LOG - fixed.size());
      auto kern = t == 0 ? k_pair_invec<R, 0> : k_pair_invec<R, LOG - 1>;  // LOG is 1 or 2
      kern<<<grid_for(nwork, kThreads, env.num_sms), kThreads, 0, env.stream>>>(re, im, nwork, make_enum(fixed, set),
                                                                             low, g);
    } else if (t < LOG + 5) {
      const uint64_t set = split(LOG + 5, fixed, low);
      const uint64_t nwork = 1ull << (n - LOG - 5 - fixed.size());
      k_pair_shfl<R><<<grid_for(nwork * 32, kThreads, env.num_sms), kThreads, 0, env.stream>>>(
          re, im, nwork, make_enum(fixed, set), t, low, g);
    } else {
      const uint64_t set = split(LOG, fixed, low);
      fixed.push_back(t);
      const uint64_t nwork = 1ull << (n - LOG - fixed.size());
      k_pair_strided<R><<<grid_for(nwork, kThreads, env.num_sms), kThreads, 0, env.stream>>>(
          re, im, nwork, make_enum(fixed, set), t, low, g);
    }
  } else {
    std::vector<uint32_t> fixed(ctrl, ctrl + nctrl);
    fixed.push_back(t);
    const uint64_t nwork = 1ull << (n - fixed.size());
    k_pair_scalar<R><<<grid_for(nwork, kThreads, env.num_sms), kThreads, 0, env.stream>>>(
        re, im, nwork, make_enum(fixed, cmask), t, g);
  }
  check_launch();
}

template <class R>
void launch_diag(const LaunchEnv& env, R* re, R* im, uint32_t n, const Sweep& s) {
  constexpr uint32_t LOG = VecT<R>::LOG;
  DiagP<R> p{};
  p.m = s.m;
  for (uint32_t j = 0; j < 6; ++j) p.q[j] = j < s.m ? s.q[j] : 63u;
  for (size_t i = 0; i < s.mat.size(); ++i) {
    p.d[2 * i] = R(s.mat[i].real());
    p.d[2 * i + 1] = R(s.mat[i].imag());
  }
  if (n >= 12) {
    // qubits whose 0-half is the identity (the "controls" the classifier found) are skipped
    std::vector<uint32_t> fixed;
    uint64_t set = 0;
    for (uint32_t i = 0; i < s.nctrl; ++i)
      if (s.ctrl[i] >= LOG) {
        fixed.push_back(s.ctrl[i]);
        set |= 1ull << s.ctrl[i];
      }
    const uint64_t nwork = 1ull << (n - LOG - fixed.size());
    k_diag<R><<<grid_for(nwork, kThreads, env.num_sms), kThreads, 0, env.stream>>>(
        re, im, nwork, make_enum(fixed, set), p);
  } else {
    const uint64_t dim = 1ull << n;
    k_diag_scalar<R><<<grid_for(dim, kThreads, env.num_sms), kThreads, 0, env.stream>>>(re, im, dim, p);
  }
  check_launch();
}

// Dense-kernel tile width per (precision, K): NCB column bits. complex128 gates of <= 3 qubits take
// 256 columns (a CTA loads, multiplies and stores its tile in turn, so a larger tile keeps more
// bytes in flight per SM; measured 2-19 % faster at 30 qubits, while wider gates measured mixed).
template <class R> constexpr int dense_ncb(int K) {
  return sizeof(R) == 4 ? 7 : (K <= 3 ? 8 : (K == 6 ? 5 : 6));
}

// Double-buffered gathers where the sweep is memory-bound (k <= 4); the compute-bound k = 5, 6
// CUDA-core tiles keep one buffer and twice the blocks per SM.
template <class R> constexpr bool dense_db(int K) { return K <= 4; }

template <class R, int K>
size_t dense_smem_bytes() {
  constexpr int M = 1 << K, NC = 1 << dense_ncb<R>(K), NB = dense_db<R>(K) ? 2 : 1;
  return size_t(2) * NB * M * NC * sizeof(R) + size_t(2) * M * M * sizeof(R) + (NC + M) * 4 + M * 8;
}

template <class R, int K>
void launch_dense_k(const LaunchEnv& env, R* re, R* im, uint32_t n, const Sweep& s, const R* ut) {
  constexpr int NCB = dense_ncb<R>(K);
  constexpr int M = 1 << K, NC = 1 << NCB, LOG = VecT<R>::LOG;
  if (n < uint32_t(K + NCB)) {
    std::vector<uint32_t> fixed(s.q, s.q + K);
    const uint64_t nb = 1ull << (n - K);
    uint32_t q[6] = {0, 0, 0, 0, 0, 0};
    for (int j = 0; j < K; ++j) q[j] = s.q[j];
    k_dense_small<R, K><<<grid_for(nb, 128, env.num_sms), 128, 0, env.stream>>>(
        re, im, nb, ut, make_enum(fixed, 0), q[0], q[1], q[2], q[3], q[4], q[5]);
    check_launch();
    return;
  }
  // tile bits: gate bits + the NCB lowest non-gate bits
  int gate_rank[64];
  for (int b = 0; b < 64; ++b) gate_rank[b] = -1;
  for (int j = 0; j < K; ++j) gate_rank[s.q[j]] = j;
  int col_rank[64];
  std::vector<uint32_t> tbits;
  int ncol = 0;
  for (uint32_t b = 0; b < n; ++b) {
    col_rank[b] = -1;
    if (gate_rank[b] >= 0) tbits.push_back(b);
    else if (ncol < NCB) {
      col_rank[b] = ncol++;
      tbits.push_back(b);
    }
  }
  auto contrib = [&](uint32_t b) -> uint32_t {
    return gate_rank[b] >= 0 ? (uint32_t(1) << gate_rank[b]) * NC : (uint32_t(1) << col_rank[b]);
  };
  DenseP p{};
  for (int j = 0; j < NCB; ++j) QSVB_REQUIRE(tbits[j] == uint32_t(j), "dense tile: low bits not contiguous");
  for (int j = 0; j < K; ++j) p.hibits[j] = tbits[NCB + j];
  for (int h = 0; h < M; ++h) {
    uint64_t off = 0;
    uint32_t d = 0;
    for (int j = 0; j < K; ++j)
      if ((h >> j) & 1) {
        off |= 1ull << p.hibits[j];
        d += contrib(p.hibits[j]);
      }
    p.hioff[h] = off;
    p.dsthi[h] = d;
  }
  for (int l = 0; l < NC; ++l) {
    uint32_t d = 0;
    for (int b = 0; b < NCB; ++b)
      if ((l >> b) & 1) d += contrib(uint32_t(b));
    p.dstlo[l] = d;
  }
  p.vecstore = 1;
  for (int b = 0; b < LOG; ++b)
    if (gate_rank[b] >= 0) p.vecstore = 0;
  const uint64_t ntiles = 1ull << (n - K - NCB);
  const size_t smem = dense_smem_bytes<R, K>();
  constexpr bool DB = dense_db<R>(K);
  QSVB_CK(cudaFuncSetAttribute(k_dense<R, K, NCB, DB>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  QSVB_CK(cudaFuncSetAttribute(k_dense<R, K, NCB, DB>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               int(cudaSharedmemCarveoutMaxShared)));
  int occ = 1;
  QSVB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_dense<R, K, NCB, DB>, kThreads, smem));
  const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(env.num_sms) * std::max(occ, 1))));
  k_dense<R, K, NCB, DB><<<grid, kThreads, smem, env.stream>>>(re, im, ntiles, ut, p);
  check_launch();
}

template <class R>
void launch_dense(const LaunchEnv& env, R* re, R* im, uint32_t n, const Sweep& s, const void* dev_mat) {
  const R* ut = static_cast<const R*>(dev_mat);
  switch (s.m) {
    case 2: launch_dense_k<R, 2>(env, re, im, n, s, ut); break;
    case 3: launch_dense_k<R, 3>(env, re, im, n, s, ut); break;
    case 4: launch_dense_k<R, 4>(env, re, im, n, s, ut); break;
    case 5: launch_dense_k<R, 5>(env, re, im, n, s, ut); break;
    case 6: launch_dense_k<R, 6>(env, re, im, n, s, ut); break;
    default: throw Error(QSVB_E_INVALID, "dense sweep arity must be 2..6");
  }
}

template <class R>
void launch_phase(const LaunchEnv& env, R* re, R* im, uint32_t n, const Sweep& s, const void* dev_terms) {
  const uint64_t dim = 1ull << n;
  const uint32_t nt = uint32_t(s.terms.size());
  if (n >= uint32_t(kIsingChunkBits)) {
    // Walsh transform of every term: theta = c0 + c1 z0 (+ c2 z1 + c3 z0 z1), index = b0 + 2 b1
    IsingP p{};
    std::vector<std::pair<uint32_t, uint32_t>> keys;
    std::vector<double> js;
    for (const PhaseTerm& t : s.terms) {
      const double* a = t.ang;
      if (t.m == 1) {
        p.c0 += 0.5 * (a[0] + a[1]);
        p.h[t.q[0]] += 0.5 * (a[0] - a[1]);
        continue;
      }
      p.c0 += 0.25 * (a[0] + a[1] + a[2] + a[3]);
      p.h[t.q[0]] += 0.25 * (a[0] - a[1] + a[2] - a[3]);
      p.h[t.q[1]] += 0.25 * (a[0] + a[1] - a[2] - a[3]);
      const double j = 0.25 * (a[0] - a[1] - a[2] + a[3]);
      const auto key = std::make_pair(std::min(t.q[0], t.q[1]), std::max(t.q[0], t.q[1]));
      const auto it = std::find(keys.begin(), keys.end(), key);
      if (it == keys.end()) {
        keys.push_back(key);
        js.push_back(j);
      } else {
        js[size_t(it - keys.begin())] += j;
      }
    }
    QSVB_REQUIRE(keys.size() <= size_t(kIsingMaxEdges), "phase polynomial has too many distinct pairs");
    p.nedges = uint32_t(keys.size());
    for (size_t e = 0; e < keys.size(); ++e) {
      p.ea[e] = uint8_t(keys[e].first);
      p.eb[e] = uint8_t(keys[e].second);
      p.J[e] = js[e];
    }
    const uint64_t nchunks = dim >> kIsingChunkBits;
    const size_t tsm = sizeof(double2) << kIsingChunkBits;
    QSVB_CK(cudaFuncSetAttribute(k_ising<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tsm)));
    k_ising<R><<<grid_for(nchunks, 1, env.num_sms, 3), kThreads, tsm, env.stream>>>(re, im, nchunks, p);
    check_launch();
    return;
  }
  const size_t smem = nt * sizeof(PhaseTermDev);
  QSVB_REQUIRE(smem <= 200 * 1024, "phase polynomial too large");
  QSVB_CK(cudaFuncSetAttribute(k_phase<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  QSVB_REQUIRE(dim % VecT<R>::N == 0, "phase sweep needs >= 2 qubits");
  k_phase<R><<<grid_for(dim / VecT<R>::N, kThreads, env.num_sms), kThreads, smem, env.stream>>>(
      re, im, dim, static_cast<const PhaseTermDev*>(dev_terms), nt);
  check_launch();
}

}  // namespace

// ------------------------------------------------------------------------------ public launchers

size_t sweep_matrix_bytes(const Sweep& s, int dtype) {
  const size_t r = dtype == QSVB_C128 ? 8 : 4;
  switch (s.kind) {
    case SK_DENSE: return 2 * r * (size_t(1) << (2 * s.m));
    case SK_DENSE_TC: return tc_matrix_bytes(s);
    case SK_PHASE: return s.terms.size() * sizeof(PhaseTermDev);
    case SK_TILE: return s.tile_blob.size();
    case SK_TC_CHAIN: return tc_chain_matrix_bytes(s);
    default: return 0;
  }
}

void pack_sweep_matrix(const Sweep& s, int dtype, void* dst) {
  if (s.kind == SK_DENSE) {
    const size_t M = size_t(1) << s.m;
    for (size_t r = 0; r < M; ++r)
      for (size_t c = 0; c < M; ++c) {
        const cd v = s.mat[r * M + c];
        const size_t o = 2 * (c * M + r);  // transposed: [s][r]
        if (dtype == QSVB_C128) {
          static_cast<double*>(dst)[o] = v.real();
          static_cast<double*>(dst)[o + 1] = v.imag();
        } else {
          static_cast<float*>(dst)[o] = float(v.real());
          static_cast<float*>(dst)[o + 1] = float(v.imag());
        }
      }
  } else if (s.kind == SK_TILE) {
    std::memcpy(dst, s.tile_blob.data(), s.tile_blob.size());
  } else if (s.kind == SK_DENSE_TC) {
    tc_pack_matrix(s, dst);
  } else if (s.kind == SK_TC_CHAIN) {
    tc_chain_pack(s, dst);
  } else if (s.kind == SK_PHASE) {
    PhaseTermDev* t = static_cast<PhaseTermDev*>(dst);
    for (size_t i = 0; i < s.terms.size(); ++i) {
      t[i].q0 = s.terms[i].q[0];
      t[i].q1 = s.terms[i].m == 2 ? s.terms[i].q[1] : 64u;
      for (int k = 0; k < 4; ++k) t[i].ang[k] = s.terms[i].ang[k];
    }
  }
}

template <class R>
void launch_sweep(const LaunchEnv& env, R* re, R* im, uint32_t n, const Sweep& s, const void* dev_mat) {
  switch (s.kind) {
    case SK_1Q: launch_pair<R>(env, re, im, n, s.target, nullptr, 0, s.mat); break;
    case SK_CTRL: launch_pair<R>(env, re, im, n, s.target, s.ctrl, s.nctrl, s.mat); break;
    case SK_DIAG: launch_diag<R>(env, re, im, n, s); break;
    case SK_PHASE: launch_phase<R>(env, re, im, n, s, dev_mat); break;
    case SK_DENSE: launch_dense<R>(env, re, im, n, s, dev_mat); break;
    case SK_DENSE_TC:
      if constexpr (sizeof(R) == 4) {
        launch_tc_dense(env, reinterpret_cast<float*>(re), reinterpret_cast<float*>(im), n, s, dev_mat);
        break;
      }
      throw Error(QSVB_E_UNSUPPORTED, "tensor-core sweeps need a complex64 state");
    case SK_TILE: launch_tile<R>(env, re, im, n, s, dev_mat); break;
    case SK_TC_CHAIN:
      if constexpr (sizeof(R) == 4) {
        launch_tc_chain(env, reinterpret_cast<float*>(re), reinterpret_cast<float*>(im), n, s, dev_mat);
        break;
      }
      throw Error(QSVB_E_UNSUPPORTED, "tensor-core chain passes need a complex64 state");
    case SK_PERMUTE: launch_permute<R>(env, re, im, n, s); break;
    case SK_NONE: break;
    default: throw Error(QSVB_E_UNSUPPORTED, "unknown sweep kind");
  }
}

template <class R> void launch_init_basis(const LaunchEnv& e, R* re, R* im, uint32_t n, uint64_t basis) {
  const size_t bytes = sizeof(R) << n;
  QSVB_CK(cudaMemsetAsync(re, 0, bytes, e.stream));
  QSVB_CK(cudaMemsetAsync(im, 0, bytes, e.stream));
  k_set_one<R><<<1, 1, 0, e.stream>>>(re, basis);
  check_launch();
}

template <class R> void launch_init_gaussian(const LaunchEnv& e, R* re, R* im, uint32_t n, uint64_t seed) {
  const uint64_t dim = 1ull << n;
  k_gaussian<R><<<grid_for(dim, kThreads, e.num_sms), kThreads, 0, e.stream>>>(re, im, dim, seed);
  check_launch();
}

template <class R> void launch_scale(const LaunchEnv& e, R* re, R* im, uint32_t n, const double* d_norm) {
  const uint64_t dim = 1ull << n;
  k_scale<R><<<grid_for(dim, kThreads, e.num_sms), kThreads, 0, e.stream>>>(re, im, dim, d_norm);
  check_launch();
}

size_t reduce_partials_needed(int num_sms) { return size_t(2) * num_sms * kReduceBlocksPerSM; }

template <class R>
void launch_reduce(const LaunchEnv& e, int op, const R* re, const R* im, const R* re2, const R* im2,
                   uint32_t n, uint64_t mask, double* partials, double* d_out) {
  const uint64_t dim = 1ull << n;
  const unsigned grid = grid_for(dim / VecT<R>::N + 1, kThreads, e.num_sms, kReduceBlocksPerSM);
  k_reduce<R><<<grid, kThreads, 0, e.stream>>>(op, re, im, re2, im2, dim, mask, partials);
  check_launch();
  k_finalize<<<1, kThreads, 0, e.stream>>>(partials, int(grid), d_out);
  check_launch();
}

template <class RA, class RB>
void launch_inner_mixed(const LaunchEnv& e, const RA* are, const RA* aim, const RB* bre, const RB* bim, uint32_t n,
                        double* partials, double* d_out) {
  const uint64_t dim = 1ull << n;
  const unsigned grid = grid_for(dim / 4 + 1, kThreads, e.num_sms, kReduceBlocksPerSM);
  k_inner_mixed<RA, RB><<<grid, kThreads, 0, e.stream>>>(are, aim, bre, bim, dim, partials);
  check_launch();
  k_finalize<<<1, kThreads, 0, e.stream>>>(partials, int(grid), d_out);
  check_launch();
}
template void launch_inner_mixed<float, double>(const LaunchEnv&, const float*, const float*, const double*,
                                                const double*, uint32_t, double*, double*);
template void launch_inner_mixed<double, float>(const LaunchEnv&, const double*, const double*, const float*,
                                                const float*, uint32_t, double*, double*);

template <class R>
void launch_probabilities(const LaunchEnv& e, const R* re, const R* im, uint64_t offset, uint64_t count,
                          void* out, int out_f64) {
  k_probs<R><<<grid_for(count, kThreads, e.num_sms), kThreads, 0, e.stream>>>(re, im, offset, count, out, out_f64);
  check_launch();
}

#define QSVB_INST(R)                                                                                   \
  template void launch_sweep<R>(const LaunchEnv&, R*, R*, uint32_t, const Sweep&, const void*);       \
  template void launch_init_basis<R>(const LaunchEnv&, R*, R*, uint32_t, uint64_t);                   \
  template void launch_init_gaussian<R>(const LaunchEnv&, R*, R*, uint32_t, uint64_t);                \
  template void launch_scale<R>(const LaunchEnv&, R*, R*, uint32_t, const double*);                   \
  template void launch_reduce<R>(const LaunchEnv&, int, const R*, const R*, const R*, const R*,       \
                                 uint32_t, uint64_t, double*, double*);                               \
  template void launch_probabilities<R>(const LaunchEnv&, const R*, const R*, uint64_t, uint64_t,     \
                                        void*, int);
QSVB_INST(float)
QSVB_INST(double)

}  // namespace qsvb
