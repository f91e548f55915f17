// Planner for tensor-core chain passes (SK_TC_CHAIN) with qubit relabelling.
//
// A chain pass works on 4096-amplitude tiles made of state bits 0..5 (so every memory access is a
// contiguous run) plus six more state bits. Which logical qubit each state bit holds is free: a
// pass may write its tile back with any permutation of the tile's 12 qubits, so the qubits a later
// pass needs can be moved onto state bits 0..5. The planner keeps that logical -> physical map:
//   1. the pass's qubit set S is the 6 qubits on state bits 0..5 plus the qubits of the first
//      pending gates (in circuit order) while S stays within 12;
//   2. every pending gate inside S that commutes past the gates it skips (disjoint qubits) is taken;
//      the taken gates are grouped by window fusion at width 6 and the first `max_mats` groups
//      become the pass's matrices (the rest stay pending), each composed in FP64 on six qubits
//      (padded with other qubits of S) ordered by state bit;
//   3. the six qubits of S needed first by the remaining gates go to state bits 0..5 for the next
//      pass; the others take the state bits those vacate (home first, qubits in place stay);
//   4. when no gate is left, permutation passes return every qubit to its own state bit.
// Gate fusion is exact, so the plan changes time, never the state beyond rounding.

#include <algorithm>
#include <cmath>
#include <numeric>

#include "qsvb_internal.h"

namespace qsvb {

namespace {

int popc(uint64_t m) { return __builtin_popcountll(m); }

// Window fusion at width 6 over a list of gates (indices into `in`), as planner.cpp's WINDOW:
// each group grows past gates it cannot take as long as every gate it takes acts on qubits
// disjoint from the gates it jumps over.
std::vector<std::vector<size_t>> window_groups(const std::vector<Gate>& in, const std::vector<size_t>& idx) {
  std::vector<char> done(idx.size(), 0);
  std::vector<std::vector<size_t>> groups;
  size_t first = 0;
  while (true) {
    while (first < idx.size() && done[first]) ++first;
    if (first == idx.size()) break;
    done[first] = 1;
    std::vector<size_t> g = {idx[first]};
    uint64_t gm = gate_mask(in[idx[first]]), blocked = 0;
    for (size_t i = first + 1; i < idx.size(); ++i) {
      if (done[i]) continue;
      const uint64_t m = gate_mask(in[idx[i]]);
      if ((m & blocked) == 0 && popc(gm | m) <= 6) {
        g.push_back(idx[i]);
        done[i] = 1;
        gm |= m;
      } else {
        blocked |= m;
        if (popc(gm) == 6 && (gm & ~blocked) == 0) break;
      }
    }
    groups.push_back(std::move(g));
  }
  return groups;
}

struct Layout {
  std::vector<uint32_t> phys;    // logical qubit -> state bit
  std::vector<uint32_t> log_at;  // state bit -> logical qubit
};

// The tile of a qubit set S (12 qubits, the six on state bits 0..5 among them): its state bits in
// ascending order.
void tile_bits_of(const Layout& lay, uint64_t S, uint32_t (&tb)[12]) {
  std::vector<uint32_t> bits;
  for (uint32_t q = 0; q < 64; ++q)
    if ((S >> q) & 1u) bits.push_back(lay.phys[q]);
  std::sort(bits.begin(), bits.end());
  QSVB_REQUIRE(bits.size() == 12, "chain planner: a tile needs 12 qubits");
  for (int i = 0; i < 12; ++i) tb[i] = bits[size_t(i)];
}

int tile_pos(const uint32_t (&tb)[12], uint32_t bit) {
  for (int i = 0; i < 12; ++i)
    if (tb[i] == bit) return i;
  return -1;
}

// Moves the qubits of S so that `low` (6 qubits of S) sit on state bits 0..5; the other qubits of S
// take the state bits of the tile those vacate: a qubit whose own state bit is among them goes home,
// qubits already in place stay. State bits 0 and 1 take two qubits of `low` that are columns of
// the pass's last matrix (`lastcols`) when there are two, so that the kernel's epilogue writes
// 16-byte vectors; among those, preferably two that are both qubits of the next pass's first
// matrix (`nextfirst`) or both not, so that its operand takes one of the two faster layouts.
// Returns the tile permutation (tile position i -> perm[i]) and updates the layout.
void relabel(Layout& lay, const uint32_t (&tb)[12], uint64_t low, uint64_t lastcols, uint64_t nextfirst,
             uint64_t finished, uint8_t (&perm)[12]) {
  std::vector<uint32_t> occ(12);
  for (int i = 0; i < 12; ++i) occ[size_t(i)] = lay.log_at[tb[i]];
  std::vector<int> dest(12, -1);
  std::vector<char> taken(12, 0);
  auto want_low = [&](int i) { return ((low >> occ[size_t(i)]) & 1u) != 0; };
  std::vector<int> pref;  // tile positions holding preferred qubits, those already on bit 0 / 1 first
  for (int i = 0; i < 2; ++i)
    if (want_low(i) && ((lastcols >> occ[size_t(i)]) & 1u)) pref.push_back(i);
  for (int i = 2; i < 12; ++i)
    if (want_low(i) && ((lastcols >> occ[size_t(i)]) & 1u)) pref.push_back(i);
  {
    std::vector<int> in_first, not_first;
    for (int i : pref) (((nextfirst >> occ[size_t(i)]) & 1u) ? in_first : not_first).push_back(i);
    if (in_first.size() >= 2 || not_first.size() >= 2) {
      // the side whose first pair keeps more qubits already on bits 0, 1 in place
      auto kept = [](const std::vector<int>& v) { return v.size() >= 2 ? int(v[0] < 2) + int(v[1] < 2) : -1; };
      pref = kept(in_first) >= kept(not_first) ? in_first : not_first;
    }
  }
  if (pref.size() >= 2) {
    for (int k = 0; k < 2; ++k)  // a preferred qubit already on bit 0 or 1 keeps it
      if (pref[size_t(k)] < 2) {
        dest[size_t(pref[size_t(k)])] = pref[size_t(k)];
        taken[size_t(pref[size_t(k)])] = 1;
      }
    for (int k = 0; k < 2; ++k) {
      const int i = pref[size_t(k)];
      if (dest[size_t(i)] >= 0) continue;
      const int t = taken[0] ? 1 : 0;
      dest[size_t(i)] = t;
      taken[size_t(t)] = 1;
    }
  }
  // qubits bound for the high side go to their own state bit when it is a free tile position
  // (fewer permutation passes at the end): those no pending gate touches first, then the others
  for (int pass = 0; pass < 2; ++pass)
    for (int i = 0; i < 12; ++i) {
      if (dest[size_t(i)] >= 0 || want_low(i)) continue;
      if ((((finished >> occ[size_t(i)]) & 1u) != 0) != (pass == 0)) continue;
      const int home = tile_pos(tb, occ[size_t(i)]);
      if (home >= 6 && !taken[size_t(home)]) {
        dest[size_t(i)] = home;
        taken[size_t(home)] = 1;
      }
    }
  // qubits already on the right side stay
  for (int i = 0; i < 12; ++i)
    if (dest[size_t(i)] < 0 && want_low(i) == (i < 6) && !taken[size_t(i)]) {
      dest[size_t(i)] = i;
      taken[size_t(i)] = 1;
    }
  // qubits leaving the low bits go home when their own bit is free in the tile
  for (int i = 0; i < 6; ++i) {
    if (dest[size_t(i)] >= 0 || want_low(i)) continue;
    const int home = tile_pos(tb, occ[size_t(i)]);
    if (home >= 6 && !taken[size_t(home)]) {
      dest[size_t(i)] = home;
      taken[size_t(home)] = 1;
    }
  }
  for (int i = 0; i < 12; ++i) {
    if (dest[size_t(i)] >= 0) continue;
    // a qubit coming to the low bits takes its own bit if that is one of them
    const int t0 = want_low(i) ? 0 : 6, t1 = want_low(i) ? 6 : 12;
    const int home = tile_pos(tb, occ[size_t(i)]);
    if (home >= t0 && home < t1 && !taken[size_t(home)]) {
      dest[size_t(i)] = home;
      taken[size_t(home)] = 1;
      continue;
    }
    for (int t = t0; t < t1; ++t)
      if (!taken[size_t(t)]) {
        dest[size_t(i)] = t;
        taken[size_t(t)] = 1;
        break;
      }
    QSVB_REQUIRE(dest[size_t(i)] >= 0, "chain planner: relabelling failed");
  }
  for (int i = 0; i < 12; ++i) {
    perm[i] = uint8_t(dest[size_t(i)]);
    const uint32_t q = occ[size_t(i)], bit = tb[dest[size_t(i)]];
    lay.phys[q] = bit;
    lay.log_at[bit] = q;
  }
}

// Moves every qubit of the tile whose own state bit is in the tile onto that bit; the others fill
// the remaining bits, low bits first. Returns the tile permutation and updates the layout.
void assign_home(Layout& lay, const uint32_t (&tb)[12], uint8_t (&perm)[12]) {
  std::vector<int> dest(12, -1);
  std::vector<char> taken(12, 0);
  std::vector<uint32_t> occ(12);
  for (int i = 0; i < 12; ++i) occ[size_t(i)] = lay.log_at[tb[i]];
  for (int i = 0; i < 12; ++i) {
    const int home = tile_pos(tb, occ[size_t(i)]);
    if (home >= 0) {
      dest[size_t(i)] = home;
      taken[size_t(home)] = 1;
    }
  }
  for (int i = 0; i < 12; ++i) {
    if (dest[size_t(i)] >= 0) continue;
    for (int t = 0; t < 12; ++t)
      if (!taken[size_t(t)]) {
        dest[size_t(i)] = t;
        taken[size_t(t)] = 1;
        break;
      }
  }
  for (int i = 0; i < 12; ++i) {
    perm[i] = uint8_t(dest[size_t(i)]);
    lay.phys[occ[size_t(i)]] = tb[dest[size_t(i)]];
    lay.log_at[tb[dest[size_t(i)]]] = occ[size_t(i)];
  }
}

// One permutation pass towards the identity layout. The misplaced qubits form cycles over state
// bits (the occupant of bit b belongs on bit c, whose occupant belongs on ...); a pass fixes every
// cycle whose high bits all fit among its six high tile bits, so the cheapest cycles go first and a
// cycle too long for what is left contributes a run of consecutive bits (all but the run's last
// occupant reach home).
Sweep restore_pass(Layout& lay, uint32_t n) {
  std::vector<char> seen(n, 0);
  std::vector<std::vector<uint32_t>> cycles;
  for (uint32_t b = 0; b < n; ++b) {
    if (seen[b] || lay.log_at[b] == b) continue;
    std::vector<uint32_t> cyc;
    for (uint32_t x = b; !seen[x]; x = lay.log_at[x]) {  // bit x's occupant belongs on bit log_at[x]
      seen[x] = 1;
      cyc.push_back(x);
    }
    cycles.push_back(std::move(cyc));
  }
  auto highs = [](const std::vector<uint32_t>& c) {
    int h = 0;
    for (uint32_t x : c) h += x >= 6;
    return h;
  };
  std::sort(cycles.begin(), cycles.end(), [&](const auto& a, const auto& b) { return highs(a) < highs(b); });
  uint64_t T = 63;
  int budget = 6;
  for (const auto& c : cycles) {
    const int h = highs(c);
    if (h <= budget) {
      for (uint32_t x : c) T |= 1ull << x;
      budget -= h;
    } else if (budget >= 2) {
      // a run of consecutive bits of the cycle (starting at a low bit when it has one)
      size_t start = 0;
      for (size_t i = 0; i < c.size(); ++i)
        if (c[i] < 6) {
          start = i;
          break;
        }
      for (size_t k = 0; k < c.size() && budget > 0; ++k) {
        const uint32_t x = c[(start + k) % c.size()];
        if (x >= 6) --budget;
        T |= 1ull << x;
      }
    }
  }
  for (uint32_t b = 6; b < n && popc(T) < 12; ++b) T |= 1ull << b;
  uint32_t tb[12];
  int k = 0;
  for (uint32_t b = 0; b < n; ++b)
    if ((T >> b) & 1u) tb[k++] = b;
  Sweep s;
  s.kind = SK_PERMUTE;
  std::copy(tb, tb + 12, s.chain_tbits);
  assign_home(lay, tb, s.chain_perm);
  return s;
}

}  // namespace

std::vector<Sweep> plan_chain(const std::vector<Gate>& in, uint32_t n, uint32_t max_mats) {
  QSVB_REQUIRE(n >= 12, "chain passes need at least 12 qubits");
  max_mats = std::max<uint32_t>(1, std::min<uint32_t>(max_mats, uint32_t(kChainMaxMats)));
  Layout lay;
  lay.phys.resize(n);
  lay.log_at.resize(n);
  std::iota(lay.phys.begin(), lay.phys.end(), 0u);
  std::iota(lay.log_at.begin(), lay.log_at.end(), 0u);
  std::vector<size_t> pending(in.size());
  std::iota(pending.begin(), pending.end(), size_t(0));
  std::vector<Sweep> out;
  // A pass's twelve qubits S (the six on state bits 0..5, `low`, then the qubits the pending gates
  // use soonest, then the lowest state bits), the pending gates it may take (`absorbed`) and its
  // matrices (window groups, at most max_mats).
  auto pass_of = [&](uint64_t low, uint64_t& S, std::vector<size_t>& absorbed) {
    S = low;
    for (size_t i : pending) {
      const uint64_t m = gate_mask(in[i]);
      if (popc(S | m) <= 12) S |= m;
      if (popc(S) == 12) break;
    }
    for (size_t i : pending) {
      if (popc(S) == 12) break;
      const Gate& g = in[i];
      for (uint32_t j = 0; j < g.m && popc(S) < 12; ++j) S |= 1ull << g.q[j];
    }
    for (uint32_t b = 6; b < n && popc(S) < 12; ++b) S |= 1ull << lay.log_at[b];
    absorbed.clear();
    uint64_t blocked = 0;
    for (size_t i : pending) {
      const uint64_t m = gate_mask(in[i]);
      if ((m & ~S) == 0 && (m & blocked) == 0) absorbed.push_back(i);
      else blocked |= m;
    }
    std::vector<std::vector<size_t>> groups = window_groups(in, absorbed);
    if (groups.size() > max_mats) groups.resize(max_mats);
    return groups;
  };
  while (!pending.empty()) {
    uint64_t low = 0;
    for (uint32_t b = 0; b < 6; ++b) low |= 1ull << lay.log_at[b];
    uint64_t S = 0;
    std::vector<size_t> absorbed;
    std::vector<std::vector<size_t>> groups = pass_of(low, S, absorbed);
    std::vector<char> kept(in.size(), 0);
    uint64_t n_gates = 0;
    for (const auto& g : groups)
      for (size_t i : g) {
        kept[i] = 1;
        ++n_gates;
      }
    uint32_t tb[12];
    tile_bits_of(lay, S, tb);
    Sweep s;
    s.kind = SK_TC_CHAIN;
    std::copy(tb, tb + 12, s.chain_tbits);
    s.chain_nmat = uint32_t(groups.size());
    s.n_gates = n_gates;
    s.chain_mats.resize(groups.size());
    for (size_t j = 0; j < groups.size(); ++j) {
      uint64_t gm = 0;
      for (size_t i : groups[j]) gm |= gate_mask(in[i]);
      // pad to six qubits of S; the first matrix prefers to hold both or neither of the qubits on
      // state bits 0 and 1 (the faster operand layouts)
      auto pad_with = [&](uint32_t q) {
        if (popc(gm) < 6 && ((S >> q) & 1u)) gm |= 1ull << q;
      };
      if (j == 0) {
        const uint32_t q0 = lay.log_at[0], q1 = lay.log_at[1];
        const bool h0 = (gm >> q0) & 1u, h1 = (gm >> q1) & 1u;
        if (h0 != h1 && popc(gm) < 6) pad_with(h0 ? q1 : q0);
      }
      std::vector<uint32_t> order;  // qubits of S by state bit; for matrix 0 bits 0, 1 last
      for (int i = 0; i < 12; ++i) order.push_back(lay.log_at[tb[i]]);
      if (j == 0 && !((gm >> lay.log_at[0]) & 1u) && !((gm >> lay.log_at[1]) & 1u))
        std::rotate(order.begin(), order.begin() + 2, order.end());
      for (uint32_t q : order) pad_with(q);
      QSVB_REQUIRE(popc(gm) == 6, "chain planner: a matrix needs six qubits");
      std::vector<uint32_t> qs;  // by ascending state bit
      for (int i = 0; i < 12; ++i)
        if ((gm >> lay.log_at[tb[i]]) & 1u) qs.push_back(lay.log_at[tb[i]]);
      // the group's gates in circuit order (window fusion only takes gates in that order)
      std::vector<const Gate*> ops;
      for (size_t i : absorbed)
        if (std::find(groups[j].begin(), groups[j].end(), i) != groups[j].end()) ops.push_back(&in[i]);
      Gate u = compose_gates(qs, ops);
      s.chain_mats[j] = std::move(u.a);
      int r = 0, c = 0;
      for (int i = 0; i < 12; ++i) {
        if ((gm >> lay.log_at[tb[i]]) & 1u) s.chain_rows[j][r++] = uint8_t(i);
        else s.chain_cols[j][c++] = uint8_t(i);
      }
    }
    std::vector<size_t> rest;
    for (size_t i : pending)
      if (!kept[i]) rest.push_back(i);
    pending.swap(rest);
    // the next pass's low qubits: those of S needed first
    uint64_t next_low = 0;
    for (size_t i : pending) {
      const Gate& g = in[i];
      for (uint32_t j = 0; j < g.m && popc(next_low) < 6; ++j)
        if ((S >> g.q[j]) & 1u) next_low |= 1ull << g.q[j];
      if (popc(next_low) == 6) break;
    }
    for (uint32_t b = 0; b < 6 && popc(next_low) < 6; ++b) next_low |= 1ull << lay.log_at[b];
    for (int i = 0; i < 12 && popc(next_low) < 6; ++i) next_low |= 1ull << lay.log_at[tb[i]];
    uint64_t lastcols = 0;  // qubits that are columns of the pass's last matrix
    {
      uint64_t lastrows = 0;
      for (int i = 0; i < 6; ++i) lastrows |= 1ull << lay.log_at[tb[s.chain_rows[s.chain_nmat - 1][i]]];
      lastcols = S & ~lastrows;
    }
    if (pending.empty()) {
      assign_home(lay, tb, s.chain_perm);  // last pass: towards the identity
    } else {
      // the next pass's first matrix (before padding), which depends only on next_low and the
      // pending gates
      uint64_t S2 = 0, nextfirst = 0;
      std::vector<size_t> absorbed2;
      const std::vector<std::vector<size_t>> g2 = pass_of(next_low, S2, absorbed2);
      if (!g2.empty())
        for (size_t i : g2[0]) nextfirst |= gate_mask(in[i]);
      uint64_t future = 0;  // qubits some pending gate touches
      for (size_t i : pending) future |= gate_mask(in[i]);
      relabel(lay, tb, next_low, lastcols, nextfirst, ~future, s.chain_perm);
    }
    tc_chain_prepare(s);
    out.push_back(std::move(s));
  }
  for (int guard = 0; guard < 64; ++guard) {
    bool identity = true;
    for (uint32_t q = 0; q < n; ++q) identity = identity && lay.phys[q] == q;
    if (identity) return out;
    out.push_back(restore_pass(lay, n));
  }
  throw Error(QSVB_E_INVALID, "chain planner: the qubit layout did not return to the identity");
}

}  // namespace qsvb
