// Oracle: a CPU restatement of qsv's own algorithms for the statevector hot path.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product library links, loads or calls this file;
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the checker
// and as the timed CPU baseline. Parity is pinned against the known answers of the reference's
// own tests (crates/qsv-core/tests/{oracle,equivalence,sampling}.rs) and against an
// independent numpy contraction; the reference itself (Rust + rayon) cannot be compiled here.
//
// What is restated, and from where (paths inside the qsv project):
//   SplitMix64 ............ crates/qsv-core/src/circuits.rs:12-48
//   gate constructors ..... crates/qsv-core/src/gate.rs:72-180
//   is_diagonal ........... crates/qsv-core/src/gate.rs:56-68
//   layout helpers ........ crates/qsv-core/src/state/layout.rs:22-86
//   RefBackend::apply ..... crates/qsv-core/src/backend/reference.rs:35-62
//   CpuBackend ............ crates/qsv-core/src/backend/cpu.rs:73-290 (OpenMP stands in for rayon,
//                           same thresholds MIN_PAIRS_LIGHT / MIN_PAIRS_HEAVY, same dispatch order)
//   fuse / build_fused .... crates/qsv-core/src/fusion.rs:39-140 (composition in the circuit's R)
//   expectation_z ......... crates/qsv-core/src/sample.rs:177-200
//   norm_sqr, probabilities crates/qsv-core/src/state/mod.rs:112-134
//
// Build: see oracle/Makefile (compiled with -ffp-contract=off so products and sums round the
// way the Rust code does: Rust never contracts a*b+c into an FMA).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <string>
#include <omp.h>

namespace {

// ---------------------------------------------------------------- SplitMix64 (circuits.rs:12-48)
struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  uint64_t below(uint64_t n) { return next() % n; }
  double unit() { return double(next() >> 11) / double(1ull << 53); }
};

// ---------------------------------------------------------------- complex in precision R
template <class R> struct C {
  R re, im;
};
template <class R> inline C<R> cadd(C<R> a, C<R> b) { return {a.re + b.re, a.im + b.im}; }
// (a+bi)(c+di) = (ac - bd) + (ad + bc)i   (complex.rs:73-80)
template <class R> inline C<R> cmul(C<R> a, C<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class R> inline bool cis_zero(C<R> a) { return a.re == R(0) && a.im == R(0); }

// A dense gate in precision R: row-major dim x dim.
template <class R> struct Gate {
  uint32_t m;
  std::vector<C<R>> a;
  size_t dim() const { return size_t(1) << m; }
  C<R> at(size_t r, size_t c) const { return a[r * dim() + c]; }
};

template <class R> Gate<R> gate_from_f64(const double* mat, uint32_t m) {
  Gate<R> g;
  g.m = m;
  size_t d = size_t(1) << m;
  g.a.resize(d * d);
  for (size_t i = 0; i < d * d; ++i) g.a[i] = {R(mat[2 * i]), R(mat[2 * i + 1])};  // Cplx::from_f64
  return g;
}

// gate.rs:56-68 — exact-zero off-diagonal test
template <class R> bool is_diagonal(const Gate<R>& g) {
  size_t d = g.dim();
  for (size_t r = 0; r < d; ++r)
    for (size_t c = 0; c < d; ++c)
      if (r != c && !cis_zero(g.at(r, c))) return false;
  return true;
}

// ---------------------------------------------------------------- layout.rs:22-86
inline uint64_t insert_zero_bit(uint64_t i, uint32_t b) {
  uint64_t left = (i >> b) << b;
  uint64_t right = i - left;
  return (left << 1) | right;
}
inline uint64_t gather_bits(uint64_t i, const uint32_t* qs, uint32_t m) {
  uint64_t g = 0;
  for (uint32_t j = 0; j < m; ++j) g |= ((i >> qs[j]) & 1ull) << j;
  return g;
}
inline uint64_t scatter_bits(uint64_t s, const uint32_t* qs, uint32_t m) {
  uint64_t x = 0;
  for (uint32_t j = 0; j < m; ++j) x |= ((s >> j) & 1ull) << qs[j];
  return x;
}
inline uint64_t insert_zero_bits(uint64_t i, const uint32_t* sorted, uint32_t m) {
  uint64_t x = i;
  for (uint32_t j = 0; j < m; ++j) x = insert_zero_bit(x, sorted[j]);
  return x;
}

// ---------------------------------------------------------------- RefBackend (reference.rs:35-62)
template <class R>
void ref_apply(R* re, R* im, uint32_t n, const Gate<R>& g, const uint32_t* qs, uint32_t m) {
  const uint64_t dim = 1ull << n;
  uint64_t qmask = 0;
  for (uint32_t j = 0; j < m; ++j) qmask |= 1ull << qs[j];
  const uint64_t nonmask = ~qmask & (dim - 1);
  const size_t gdim = g.dim();
  std::vector<C<R>> out(dim);
  for (uint64_t r = 0; r < dim; ++r) {
    uint64_t fixed = r & nonmask;
    uint64_t gr = gather_bits(r, qs, m);
    C<R> acc{R(0), R(0)};
    for (size_t gc = 0; gc < gdim; ++gc) {
      uint64_t col = fixed | scatter_bits(gc, qs, m);
      acc = cadd(acc, cmul(g.at(gr, gc), C<R>{re[col], im[col]}));
    }
    out[r] = acc;
  }
  for (uint64_t i = 0; i < dim; ++i) {
    re[i] = out[i].re;
    im[i] = out[i].im;
  }
}

// ---------------------------------------------------------------- CpuBackend (cpu.rs:73-290)
constexpr uint64_t kMinPairsLight = 1ull << 16;  // cpu.rs:44
constexpr uint64_t kMinPairsHeavy = 1ull << 12;  // cpu.rs:45

template <class R>
inline void one_qubit_block(R* rl, R* il, R* rh, R* ih, uint64_t len, const C<R> g[4]) {
  for (uint64_t i = 0; i < len; ++i) {
    C<R> x0{rl[i], il[i]}, x1{rh[i], ih[i]};
    C<R> y0 = cadd(cmul(g[0], x0), cmul(g[1], x1));
    C<R> y1 = cadd(cmul(g[2], x0), cmul(g[3], x1));
    rl[i] = y0.re;
    il[i] = y0.im;
    rh[i] = y1.re;
    ih[i] = y1.im;
  }
}

template <class R>
inline void diag_chunk(uint64_t base, R* rc, R* ic, uint64_t len, const C<R>* diag,
                       const uint32_t* qs, uint32_t m) {
  for (uint64_t o = 0; o < len; ++o) {
    uint64_t s = gather_bits(base + o, qs, m);
    R dr = diag[s].re, di = diag[s].im;
    R xr = rc[o], xi = ic[o];
    rc[o] = dr * xr - di * xi;
    ic[o] = dr * xi + di * xr;
  }
}

template <class R>
void cpu_apply_diagonal(R* re, R* im, uint32_t n, const Gate<R>& g, const uint32_t* qs,
                        uint32_t m, bool parallel) {
  C<R> diag[64];
  for (size_t s = 0; s < g.dim(); ++s) diag[s] = g.at(s, s);
  const uint64_t dim = 1ull << n;
  if (parallel && dim >= (kMinPairsLight << 1)) {
    uint64_t nthreads = std::max(1, omp_get_max_threads());
    uint64_t chunk = std::max<uint64_t>(dim / (4 * nthreads), 1u << 10);
    int64_t nchunks = int64_t((dim + chunk - 1) / chunk);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nchunks; ++c) {
      uint64_t b = uint64_t(c) * chunk;
      uint64_t len = std::min(chunk, dim - b);
      diag_chunk(b, re + b, im + b, len, diag, qs, m);
    }
    return;
  }
  diag_chunk<R>(0, re, im, dim, diag, qs, m);
}

template <class R>
void cpu_apply_1q(R* re, R* im, uint32_t n, const Gate<R>& g, uint32_t q, bool parallel) {
  const C<R> gg[4] = {g.at(0, 0), g.at(0, 1), g.at(1, 0), g.at(1, 1)};
  const uint64_t half = 1ull << q, block = half << 1, dim = 1ull << n;
  const int64_t nblocks = int64_t(dim / block);
  if (parallel && (dim >> 1) >= kMinPairsLight) {
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < nblocks; ++b) {
      uint64_t o = uint64_t(b) * block;
      one_qubit_block(re + o, im + o, re + o + half, im + o + half, half, gg);
    }
    return;
  }
  for (int64_t b = 0; b < nblocks; ++b) {
    uint64_t o = uint64_t(b) * block;
    one_qubit_block(re + o, im + o, re + o + half, im + o + half, half, gg);
  }
}

template <class R>
inline void mq_block(R* re, R* im, const Gate<R>& g, const uint32_t* qs, uint32_t m,
                     uint64_t base, size_t sub) {
  C<R> amp[64];
  for (size_t s = 0; s < sub; ++s) {
    uint64_t idx = base | scatter_bits(s, qs, m);
    amp[s] = {re[idx], im[idx]};
  }
  for (size_t r = 0; r < sub; ++r) {
    C<R> acc{R(0), R(0)};
    for (size_t c = 0; c < sub; ++c) acc = cadd(acc, cmul(g.a[r * sub + c], amp[c]));
    uint64_t idx = base | scatter_bits(r, qs, m);
    re[idx] = acc.re;
    im[idx] = acc.im;
  }
}

template <class R>
void cpu_apply_mq(R* re, R* im, uint32_t n, const Gate<R>& g, const uint32_t* qs, uint32_t m,
                  bool parallel) {
  const size_t sub = size_t(1) << m;
  uint32_t sorted[6];
  std::copy(qs, qs + m, sorted);
  std::sort(sorted, sorted + m);
  const uint64_t dim = 1ull << n, blocks = dim >> m;
  if (parallel && (dim >> 1) >= kMinPairsHeavy && blocks > 1) {
#pragma omp parallel for schedule(static)
    for (int64_t o = 0; o < int64_t(blocks); ++o)
      mq_block(re, im, g, qs, m, insert_zero_bits(uint64_t(o), sorted, m), sub);
    return;
  }
  for (uint64_t o = 0; o < blocks; ++o) mq_block(re, im, g, qs, m, insert_zero_bits(o, sorted, m), sub);
}

template <class R>
void cpu_apply(R* re, R* im, uint32_t n, const Gate<R>& g, const uint32_t* qs, uint32_t m,
               bool parallel) {
  if (is_diagonal(g))
    cpu_apply_diagonal(re, im, n, g, qs, m, parallel);
  else if (m == 1)
    cpu_apply_1q(re, im, n, g, qs[0], parallel);
  else
    cpu_apply_mq(re, im, n, g, qs, m, parallel);
}

template <class R>
void apply_any(int engine, R* re, R* im, uint32_t n, const Gate<R>& g, const uint32_t* qs,
               uint32_t m) {
  if (engine == 0)
    ref_apply(re, im, n, g, qs, m);
  else
    cpu_apply(re, im, n, g, qs, m, engine == 2);
}

// ---------------------------------------------------------------- fusion.rs:39-140
inline uint64_t gather_local(uint64_t idx, const std::vector<uint32_t>& local) {
  uint64_t s = 0;
  for (size_t j = 0; j < local.size(); ++j) s |= ((idx >> local[j]) & 1ull) << j;
  return s;
}
inline uint64_t set_local(uint64_t idx, const std::vector<uint32_t>& local, uint64_t sub) {
  uint64_t x = idx;
  for (size_t j = 0; j < local.size(); ++j) {
    uint64_t bit = (sub >> j) & 1ull;
    x = (x & ~(1ull << local[j])) | (bit << local[j]);
  }
  return x;
}

template <class R> struct Op {
  Gate<R> g;
  std::vector<uint32_t> qs;
};

template <class R>
Gate<R> build_fused(const std::vector<uint32_t>& q, const std::vector<const Op<R>*>& ops) {
  const size_t dim = size_t(1) << q.size();
  std::vector<C<R>> mat(dim * dim, C<R>{R(0), R(0)});
  for (size_t i = 0; i < dim; ++i) mat[i * dim + i] = {R(1), R(0)};
  for (const Op<R>* op : ops) {
    std::vector<uint32_t> local;
    for (uint32_t x : op->qs) local.push_back(uint32_t(std::find(q.begin(), q.end(), x) - q.begin()));
    const size_t nsub = size_t(1) << op->qs.size();
    std::vector<C<R>> nw(dim * dim, C<R>{R(0), R(0)});
    for (size_t r = 0; r < dim; ++r) {
      uint64_t rs = gather_local(r, local);
      for (size_t ks = 0; ks < nsub; ++ks) {
        C<R> e = op->g.at(rs, ks);
        if (cis_zero(e)) continue;
        uint64_t k = set_local(r, local, ks);
        for (size_t c = 0; c < dim; ++c) nw[r * dim + c] = cadd(nw[r * dim + c], cmul(e, mat[k * dim + c]));
      }
    }
    mat.swap(nw);
  }
  Gate<R> g;
  g.m = uint32_t(q.size());
  g.a = std::move(mat);
  return g;
}

template <class R>
void flush_group(std::vector<Op<R>>& out, std::vector<uint32_t>& gq, std::vector<const Op<R>*>& gops) {
  if (gops.size() == 1) {
    out.push_back(*gops[0]);
  } else if (gops.size() > 1) {
    std::vector<uint32_t> q = gq;
    std::sort(q.begin(), q.end());
    Op<R> f;
    f.g = build_fused(q, gops);
    f.qs = q;
    out.push_back(std::move(f));
  }
  gq.clear();
  gops.clear();
}

template <class R> std::vector<Op<R>> fuse(const std::vector<Op<R>>& ops, uint32_t max_qubits) {
  const uint32_t mx = std::max<uint32_t>(max_qubits, 1);
  std::vector<Op<R>> out;
  std::vector<uint32_t> gq;
  std::vector<const Op<R>*> gops;
  for (const Op<R>& op : ops) {
    if (op.qs.size() > mx) {
      flush_group(out, gq, gops);
      out.push_back(op);
      continue;
    }
    std::vector<uint32_t> uni = gq;
    for (uint32_t x : op.qs)
      if (std::find(uni.begin(), uni.end(), x) == uni.end()) uni.push_back(x);
    if (gops.empty()) {
      gq = op.qs;
      gops.push_back(&op);
    } else if (uni.size() <= mx) {
      gq = uni;
      gops.push_back(&op);
    } else {
      flush_group(out, gq, gops);
      gq = op.qs;
      gops.push_back(&op);
    }
  }
  flush_group(out, gq, gops);
  return out;
}

template <class R>
std::vector<Op<R>> unpack_ops(size_t nops, const uint32_t* arity, const uint32_t* qubits,
                              const double* mats) {
  std::vector<Op<R>> ops(nops);
  size_t qo = 0, mo = 0;
  for (size_t i = 0; i < nops; ++i) {
    uint32_t m = arity[i];
    ops[i].g = gate_from_f64<R>(mats + mo, m);
    ops[i].qs.assign(qubits + qo, qubits + qo + m);
    qo += m;
    mo += 2 * (size_t(1) << (2 * m));
  }
  return ops;
}

// ---------------------------------------------------------------- gate.rs:72-180
void put(double* o, size_t i, double re, double im) {
  o[2 * i] = re;
  o[2 * i + 1] = im;
}

void controlled_1q(const double* u, double* out) {  // gate.rs:72-87, qs = [control, target]
  std::fill(out, out + 32, 0.0);
  put(out, 0, 1, 0);
  put(out, 2 * 4 + 2, 1, 0);
  for (int to = 0; to < 2; ++to)
    for (int ti = 0; ti < 2; ++ti) {
      int row = 1 + 2 * to, col = 1 + 2 * ti;
      put(out, size_t(row * 4 + col), u[2 * (to * 2 + ti)], u[2 * (to * 2 + ti) + 1]);
    }
}

bool gate_by_name(const char* name, double th, double* o, uint32_t* m) {
  const double r2 = 0.70710678118654752440;  // FRAC_1_SQRT_2
  std::string n(name);
  double tmp[8];
  *m = 1;
  std::fill(o, o + 8, 0.0);
  if (n == "h") { put(o, 0, r2, 0); put(o, 1, r2, 0); put(o, 2, r2, 0); put(o, 3, -r2, 0); }
  else if (n == "x") { put(o, 1, 1, 0); put(o, 2, 1, 0); }
  else if (n == "y") { put(o, 1, 0, -1); put(o, 2, 0, 1); }
  else if (n == "z") { put(o, 0, 1, 0); put(o, 3, -1, 0); }
  else if (n == "s") { put(o, 0, 1, 0); put(o, 3, 0, 1); }
  else if (n == "t") { put(o, 0, 1, 0); put(o, 3, r2, r2); }
  else if (n == "sx") { put(o, 0, .5, .5); put(o, 1, .5, -.5); put(o, 2, .5, -.5); put(o, 3, .5, .5); }
  else if (n == "rx") { double s = std::sin(th * .5), c = std::cos(th * .5);
    put(o, 0, c, 0); put(o, 1, 0, -s); put(o, 2, 0, -s); put(o, 3, c, 0); }
  else if (n == "ry") { double s = std::sin(th * .5), c = std::cos(th * .5);
    put(o, 0, c, 0); put(o, 1, -s, 0); put(o, 2, s, 0); put(o, 3, c, 0); }
  else if (n == "rz") { double s = std::sin(th * .5), c = std::cos(th * .5);
    put(o, 0, c, -s); put(o, 3, c, s); }
  else if (n == "phase") { double s = std::sin(th), c = std::cos(th); put(o, 0, 1, 0); put(o, 3, c, s); }
  else {
    *m = 2;
    std::fill(o, o + 32, 0.0);
    std::fill(tmp, tmp + 8, 0.0);
    if (n == "cx") { put(tmp, 1, 1, 0); put(tmp, 2, 1, 0); controlled_1q(tmp, o); }
    else if (n == "cz") { put(tmp, 0, 1, 0); put(tmp, 3, -1, 0); controlled_1q(tmp, o); }
    else if (n == "cphase") { double s = std::sin(th), c = std::cos(th);
      put(tmp, 0, 1, 0); put(tmp, 3, c, s); controlled_1q(tmp, o); }
    else if (n == "swap") { put(o, 0, 1, 0); put(o, 6, 1, 0); put(o, 9, 1, 0); put(o, 15, 1, 0); }
    else if (n == "rzz") {
      for (int idx = 0; idx < 4; ++idx) {
        int parity = (idx & 1) ^ ((idx >> 1) & 1);
        double zz = parity == 0 ? 1.0 : -1.0;
        double a = -0.5 * th * zz;
        put(o, size_t(idx * 4 + idx), std::cos(a), std::sin(a));
      }
    } else return false;
  }
  return true;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------ RNG
uint64_t orc_splitmix_next(uint64_t* state) {
  SplitMix64 r{*state};
  uint64_t v = r.next();
  *state = r.s;
  return v;
}
double orc_splitmix_unit(uint64_t* state) {
  SplitMix64 r{*state};
  double v = r.unit();
  *state = r.s;
  return v;
}
uint64_t orc_splitmix_below(uint64_t* state, uint64_t n) {
  SplitMix64 r{*state};
  uint64_t v = r.below(n);
  *state = r.s;
  return v;
}

// ------------------------------------------------------------------ gates
// Writes the gate's row-major interleaved (re, im) FP64 matrix; returns 0 or -1 for an unknown name.
int orc_gate(const char* name, double theta, double* out, uint32_t* m) {
  return gate_by_name(name, theta, out, m) ? 0 : -1;
}

int orc_is_diagonal(const double* mat, uint32_t m) {
  return is_diagonal(gate_from_f64<double>(mat, m)) ? 1 : 0;
}

// ------------------------------------------------------------------ layout helpers
uint64_t orc_insert_zero_bit(uint64_t i, uint32_t b) { return insert_zero_bit(i, b); }
uint64_t orc_insert_zero_bits(uint64_t i, const uint32_t* sorted, uint32_t m) {
  return insert_zero_bits(i, sorted, m);
}
uint64_t orc_gather_bits(uint64_t i, const uint32_t* qs, uint32_t m) { return gather_bits(i, qs, m); }
uint64_t orc_scatter_bits(uint64_t s, const uint32_t* qs, uint32_t m) { return scatter_bits(s, qs, m); }

void orc_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int orc_max_threads(void) { return omp_get_max_threads(); }

// ------------------------------------------------------------------ apply
// engine: 0 = RefBackend, 1 = CpuBackend::serial, 2 = CpuBackend::parallel.
// dtype:  0 = f32 state (float re/im), 1 = f64 state. Matrices arrive as FP64 and are rounded to R
// exactly as Cplx::from_f64 does.
int orc_apply(int engine, int dtype, uint32_t n, void* re, void* im, const double* mat,
              const uint32_t* qs, uint32_t m) {
  if (m < 1 || m > 6 || m > n) return -1;
  if (dtype == 1)
    apply_any(engine, (double*)re, (double*)im, n, gate_from_f64<double>(mat, m), qs, m);
  else
    apply_any(engine, (float*)re, (float*)im, n, gate_from_f64<float>(mat, m), qs, m);
  return 0;
}

// Apply a flattened circuit: op i has arity[i] qubits (concatenated in `qubits`) and a
// 2^m x 2^m interleaved FP64 matrix (concatenated in `mats`).
int orc_run(int engine, int dtype, uint32_t n, void* re, void* im, size_t nops,
            const uint32_t* arity, const uint32_t* qubits, const double* mats) {
  size_t qo = 0, mo = 0;
  for (size_t i = 0; i < nops; ++i) {
    int rc = orc_apply(engine, dtype, n, re, im, mats + mo, qubits + qo, arity[i]);
    if (rc) return rc;
    qo += arity[i];
    mo += 2 * (size_t(1) << (2 * arity[i]));
  }
  return 0;
}

// Reference fuse in precision R (dtype 0 = f32, 1 = f64). Writes the fused ops; fused matrices
// are written back as FP64 (exact widening of R). Returns the number of fused ops, or
// -(needed doubles) when out_mats_cap is too small.
long orc_fuse(int dtype, uint32_t max_qubits, size_t nops, const uint32_t* arity,
              const uint32_t* qubits, const double* mats, uint32_t* out_arity,
              uint32_t* out_qubits, double* out_mats, size_t out_mats_cap) {
  auto emit = [&](auto&& fused) -> long {
    size_t need = 0;
    for (auto& op : fused) need += 2 * op.g.a.size();
    if (need > out_mats_cap) return -long(need);
    size_t qo = 0, mo = 0;
    for (size_t i = 0; i < fused.size(); ++i) {
      out_arity[i] = uint32_t(fused[i].qs.size());
      for (uint32_t q : fused[i].qs) out_qubits[qo++] = q;
      for (auto& c : fused[i].g.a) {
        out_mats[mo++] = double(c.re);
        out_mats[mo++] = double(c.im);
      }
    }
    return long(fused.size());
  };
  if (dtype == 1) return emit(fuse(unpack_ops<double>(nops, arity, qubits, mats), max_qubits));
  return emit(fuse(unpack_ops<float>(nops, arity, qubits, mats), max_qubits));
}

// ------------------------------------------------------------------ reductions
// state/mod.rs:130-134 — |psi_i|^2 in R
void orc_probabilities(int dtype, const void* re, const void* im, uint64_t len, void* out) {
  if (dtype == 1) {
    const double *r = (const double*)re, *i = (const double*)im;
    double* o = (double*)out;
    for (uint64_t k = 0; k < len; ++k) o[k] = r[k] * r[k] + i[k] * i[k];
  } else {
    const float *r = (const float*)re, *i = (const float*)im;
    float* o = (float*)out;
    for (uint64_t k = 0; k < len; ++k) o[k] = r[k] * r[k] + i[k] * i[k];
  }
}

// state/mod.rs:112-118 — sequential sum accumulated in R, returned widened to f64
double orc_norm_sqr(int dtype, const void* re, const void* im, uint64_t len) {
  if (dtype == 1) {
    const double *r = (const double*)re, *i = (const double*)im;
    double s = 0;
    for (uint64_t k = 0; k < len; ++k) s = s + r[k] * r[k] + i[k] * i[k];
    return s;
  }
  const float *r = (const float*)re, *i = (const float*)im;
  float s = 0;
  for (uint64_t k = 0; k < len; ++k) s = s + r[k] * r[k] + i[k] * i[k];
  return double(s);
}

// sample.rs:177-200 — sum_i p_i (-1)^popcount(i & mask) in f64 (serial order)
double orc_expectation_z(int dtype, const void* probs, uint64_t len, uint64_t mask) {
  double s = 0;
  for (uint64_t k = 0; k < len; ++k) {
    double p = dtype == 1 ? ((const double*)probs)[k] : double(((const float*)probs)[k]);
    s += (__builtin_popcountll(k & mask) & 1) ? -p : p;
  }
  return s;
}

}  // extern "C"
