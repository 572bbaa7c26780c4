// Netlist + fault list -> device plan (see fsimb_plan.h).
#include "fsimb_plan.h"

#include <algorithm>
#include <array>
#include <cstring>
#include <functional>

namespace fsimb {

namespace {

// Inputs an element's evaluation reads: INV, CLKBUF and PO use their first
// input only (fsim/simulation.cpp:979-983, 1062-1067, 1074-1077).
uint32_t eff_fanin(const Netlist& nl, uint32_t e) {
  uint32_t nf = nl.fanin_count(e);
  const uint8_t t = nl.type[e];
  if (t == G_INV || t == G_CLKBUF || t == G_PO) nf = std::min<uint32_t>(nf, 1);
  return nf;
}

}  // namespace

uint32_t gate_class(uint8_t type, uint32_t nf) {
  const uint32_t fam = gate_family(type);
  if (fam == 0 && nf >= 1 && nf <= 4) return nf - 1;
  if (fam == 1 && nf >= 2 && nf <= 4) return 4 + nf - 2;
  if (fam == 2 && nf == 3) return 7;
  return kClassGeneric;
}

uint32_t plain_class(uint8_t t, uint32_t nf) {
  if (nf == 1) {
    switch (t) {
      case G_AND: case G_OR: case G_XOR: case G_CLKBUF: return kPBuf;
      case G_INV: case G_NAND: case G_NOR: case G_XNOR: return kPInv;
      default: return kPlainClasses;
    }
  }
  if (nf != 2 && nf != 3) return kPlainClasses;
  const uint32_t base = nf == 2 ? kPAnd2 : kPAnd3;
  switch (t) {
    case G_AND: return base + 0;
    case G_NAND: return base + 1;
    case G_OR: return base + 2;
    case G_NOR: return base + 3;
    case G_XOR: return base + 4;
    case G_XNOR: return base + 5;
    default: return kPlainClasses;
  }
}

uint32_t gate_family(uint8_t t) {
  switch (t) {
    case G_XOR:
    case G_XNOR: return 1;
    case G_MUX: return 2;
    default: return 0;
  }
}

void build_circuit_plan(const Netlist& nl, CircuitPlan& C) {
  C = CircuitPlan();
  Plan& P = C.base;
  const uint32_t N = nl.N;
  P.N = N;
  P.n_pi = (uint32_t)nl.n_pi;
  P.n_gates = (uint32_t)nl.n_gates;
  P.n_po = (uint32_t)nl.n_po;
  P.n_levels = nl.n_levels;
  P.level_off = nl.level_off;
  const uint32_t po_begin = P.n_pi + P.n_gates;
  P.max_gate_level = P.n_gates ? nl.level[po_begin - 1] : 0;
  for (uint32_t l = 0; l < nl.n_levels; ++l)
    P.max_level_width = std::max<uint32_t>(P.max_level_width, nl.level_off[l + 1] - nl.level_off[l]);

  // Per-element fanout facts.
  C.mux_below.assign(N, 0);
  P.po_drv.assign(N, 0);
  P.gate_fo.assign(N, 0);
  P.maxfo_level.assign(N, 0);
  for (uint32_t e = 0; e < N; ++e) {
    for (uint32_t k = nl.fo_off[e]; k < nl.fo_off[e + 1]; ++k) {
      uint32_t c = nl.fo_idx[k];
      if (nl.type[c] == G_PO) {
        P.po_drv[e] = 1;
      } else {
        P.gate_fo[e] = 1;
        P.maxfo_level[e] = std::max(P.maxfo_level[e], nl.level[c]);
      }
    }
    P.has_mux |= nl.type[e] == G_MUX;
  }
  for (int64_t e = (int64_t)N - 1; e >= 0; --e) {
    uint8_t hb = 0;
    for (uint32_t k = nl.fo_off[e]; k < nl.fo_off[e + 1]; ++k) {
      uint32_t c = nl.fo_idx[k];
      hb |= (nl.type[c] == G_MUX) | C.mux_below[c];
    }
    C.mux_below[e] = hb;
  }

  // Peak number of live values (interval graph of [level, highest consumer
  // level]); the schedule may need a few more to honour slot residues.
  {
    std::vector<int64_t> delta(nl.n_levels + 2, 0);
    for (uint32_t e = 0; e < N; ++e)
      if (P.gate_fo[e]) {
        delta[nl.level[e]]++;
        delta[P.maxfo_level[e] + 1]--;
      }
    int64_t live = 0;
    for (uint32_t l = 0; l < nl.n_levels; ++l) {
      live += delta[l];
      P.max_live = std::max<uint32_t>(P.max_live, (uint32_t)live);
    }
  }

  // FFR roots: an element with exactly one consumer belongs to the FFR of that
  // consumer; the members of each FFR, element-descending (consumer first).
  C.root.resize(N);
  for (int64_t e = (int64_t)N - 1; e >= 0; --e) {
    uint32_t fo = nl.fo_off[e + 1] - nl.fo_off[e];
    if (nl.type[e] == G_PO || fo != 1)
      C.root[e] = (uint32_t)e;
    else
      C.root[e] = C.root[nl.fo_idx[nl.fo_off[e]]];
  }
  C.ffr_off.assign(N + 1, 0);
  for (uint32_t e = 0; e < N; ++e)
    if (C.root[e] != e) C.ffr_off[C.root[e] + 1]++;
  for (uint32_t r = 0; r < N; ++r) C.ffr_off[r + 1] += C.ffr_off[r];
  C.ffr_mem.resize(C.ffr_off[N]);
  C.ffr_local.assign(N, 0);
  {
    std::vector<uint32_t> fill(C.ffr_off.begin(), C.ffr_off.end() - 1);
    for (int64_t e = (int64_t)N - 1; e >= 0; --e) {
      const uint32_t r = C.root[e];
      if (r == (uint32_t)e) continue;
      const uint32_t k = nl.fo_off[e];
      C.ffr_local[e] = fill[r] - C.ffr_off[r];
      C.ffr_mem[fill[r]++] = MemberRec{(uint32_t)e, nl.fo_idx[k], nl.fo_pin[k], 0};
    }
  }

  // Algorithmic bytes of one gate-word evaluation: its fanin words read and
  // its output word written, 8 * (fanin + 1).  A sweep evaluates the gates
  // that feed a gate or a PO; gates that feed nothing cannot change a PO.
  P.nfp_prefix.assign(N + 1, 0);
  P.eval_prefix.assign(N + 1, 0);
  for (uint32_t e = 0; e < N; ++e) {
    const bool ev = e >= P.n_pi && (P.gate_fo[e] || P.po_drv[e]);
    const uint32_t nf = ev ? eff_fanin(nl, e) : 0;
    P.nfp_prefix[e + 1] = P.nfp_prefix[e] + (ev ? 8ull * (nf + 1) : 0);
    P.eval_prefix[e + 1] = P.eval_prefix[e] + (ev ? 1 : 0);
  }
}

void build_fault_plan(const Netlist& nl, const CircuitPlan& C, const std::vector<Fault>& faults,
                      Plan& P) {
  const Plan& B = C.base;
  P = Plan();
  P.N = B.N;
  P.n_pi = B.n_pi;
  P.n_gates = B.n_gates;
  P.n_po = B.n_po;
  P.n_levels = B.n_levels;
  P.level_off = B.level_off;
  P.max_gate_level = B.max_gate_level;
  P.max_level_width = B.max_level_width;
  P.max_live = B.max_live;
  P.has_mux = B.has_mux;
  auto reaches_po = [&](uint32_t x) {
    return (nl.type[x] == G_PO || B.po_drv[x]) ? kInjReachesPo : 0u;
  };
  auto is_exact = [&](const Fault& ft) {
    return ft.pin == 0 ? (bool)C.mux_below[ft.site]
                       : (nl.type[ft.site] == G_MUX || C.mux_below[ft.site]);
  };

  // Traced faults grouped by FFR root (fault order within a root), roots in
  // topological order so neighbouring warps touch neighbouring data.
  std::vector<std::pair<uint32_t, uint32_t>> rf;  // (root, fault)
  rf.reserve(faults.size());
  for (uint32_t f = 0; f < faults.size(); ++f)
    if (!is_exact(faults[f])) rf.emplace_back(C.root[faults[f].site], f);
  std::stable_sort(rf.begin(), rf.end(),
                   [](const std::pair<uint32_t, uint32_t>& a, const std::pair<uint32_t, uint32_t>& b) {
                     return a.first < b.first;
                   });
  for (size_t i = 0; i < rf.size();) {
    const uint32_t r = rf[i].first;
    RootRec rr{};
    rr.root = r;
    if (nl.type[r] == G_PO || B.po_drv[r])
      rr.obs = kObsOne;
    else if (!B.gate_fo[r])
      rr.obs = kObsZero;
    else {
      rr.obs = (uint32_t)P.sweeps.size();
      P.sweeps.push_back(InjRec{r, 0, reaches_po(r), 0});
      P.sweep_root.push_back((uint32_t)P.roots.size());
    }
    rr.mem_begin = (uint32_t)P.members.size();
    // a member's slot is its index in members; its consumer is the root
    // (patched below, once the number of members is known) or a member of
    // the same FFR listed before it
    for (uint32_t k = C.ffr_off[r]; k < C.ffr_off[r + 1]; ++k) {
      MemberRec m = C.ffr_mem[k];
      m.p_slot = m.p == r ? kNoSlot : rr.mem_begin + C.ffr_local[m.p];
      P.members.push_back(m);
    }
    rr.mem_end = (uint32_t)P.members.size();
    rr.flt_begin = (uint32_t)P.traced.size();
    for (; i < rf.size() && rf[i].first == r; ++i) {
      const Fault& ft = faults[rf[i].second];
      P.traced.push_back(TracedRec{rf[i].second, ft.site, ft.pin, ft.value});
      P.traced_slot.push_back(ft.site == r ? kNoSlot : rr.mem_begin + C.ffr_local[ft.site]);
    }
    rr.flt_end = (uint32_t)P.traced.size();
    P.roots.push_back(rr);
  }
  // root slots follow the members
  const uint32_t n_mem = (uint32_t)P.members.size();
  for (uint32_t ri = 0; ri < P.roots.size(); ++ri) {
    RootRec& rr = P.roots[ri];
    rr.slot = n_mem + ri;
    for (uint32_t k = rr.mem_begin; k < rr.mem_end; ++k)
      if (P.members[k].p_slot == kNoSlot) P.members[k].p_slot = rr.slot;
    for (uint32_t k = rr.flt_begin; k < rr.flt_end; ++k)
      if (P.traced_slot[k] == kNoSlot) P.traced_slot[k] = rr.slot;
  }
  P.n_stem_sweeps = (uint32_t)P.sweeps.size();
  for (uint32_t f = 0; f < faults.size(); ++f) {
    const Fault& ft = faults[f];
    if (!is_exact(ft)) continue;
    P.sweeps.push_back(InjRec{ft.site, ft.pin, kInjStuck | reaches_po(ft.site), ft.value});
    P.exact_fault.push_back(f);
  }

  const uint32_t gates_end = nl.level_off[std::min(P.max_gate_level + 1, nl.n_levels)];
  for (auto& s : P.sweeps) {
    uint32_t L0 = nl.level[s.elem] + 1;
    if (L0 <= P.max_gate_level) {
      P.dense_sweep_gates += B.eval_prefix[gates_end] - B.eval_prefix[nl.level_off[L0]];
      P.dense_sweep_bytes += B.nfp_prefix[gates_end] - B.nfp_prefix[nl.level_off[L0]];
    }
  }
}

void build_plan(const Netlist& nl, const std::vector<Fault>& faults, Plan& P) {
  CircuitPlan C;
  build_circuit_plan(nl, C);
  build_fault_plan(nl, C, faults, P);
  P.maxfo_level = std::move(C.base.maxfo_level);
  P.gate_fo = std::move(C.base.gate_fo);
  P.po_drv = std::move(C.base.po_drv);
  P.nfp_prefix = std::move(C.base.nfp_prefix);
  P.eval_prefix = std::move(C.base.eval_prefix);
}

// ---------------------------------------------------------------- schedule
namespace {

struct SlotPool {
  uint32_t G;
  uint32_t next_block = 0;
  std::vector<std::vector<uint32_t>> free;  // per residue
  explicit SlotPool(uint32_t g) : G(g), free(g) {}
  uint32_t alloc(uint32_t r) {
    if (free[r].empty()) {
      for (uint32_t q = 0; q < G; ++q) free[q].push_back(next_block * G + q);
      ++next_block;
    }
    uint32_t s = free[r].back();
    free[r].pop_back();
    return s;
  }
  void release(uint32_t s) { free[s % G].push_back(s); }
};

}  // namespace

void build_schedule(const Netlist& nl, const Plan& P, uint32_t G, Schedule& S) {
  S = Schedule();
  S.G = G;
  const uint32_t N = nl.N;
  std::vector<uint32_t> slot(N, kNoSlot);
  SlotPool pool(G);
  std::vector<std::vector<uint32_t>> release(nl.n_levels + 2);
  // PIs: residues round robin.
  uint32_t rr = 0;
  for (uint32_t e = nl.level_off[0]; e < nl.level_off[1]; ++e) {
    if (!P.gate_fo[e]) continue;
    slot[e] = pool.alloc(rr++ % G);
    release[P.maxfo_level[e] + 1].push_back(slot[e]);
  }
  auto nf_of = [&](uint32_t e) { return std::min<uint32_t>(eff_fanin(nl, e), 4); };
  // Classes by (gate family, fan-in): a warp runs one code path.  The AND
  // family (AND, NAND, OR, NOR, INV, CLKBUF) is io ^ AND(in ^ ii), the XOR
  // family io ^ XOR(in); MUX is its own family.
  auto cls_of = [&](uint32_t e) { return gate_family(nl.type[e]) * 8 + nf_of(e); };
  // Record position k of element e reads its fanin perm[e][k]: the AND and
  // XOR families are commutative, so the grouper may reorder their fanins
  // (pin faults and FFR tracing use the netlist's pin order, not the
  // records); MUX keeps its order.
  std::vector<std::array<uint8_t, 4>> perm(N, std::array<uint8_t, 4>{0, 1, 2, 3});
  auto res_in = [&](uint32_t e, uint32_t k) { return slot[nl.fi_idx[nl.fi_off[e] + k]] % G; };
  // permutations of 2, 3 and 4 inputs
  static const uint8_t kPerm2[2][4] = {{0, 1, 2, 3}, {1, 0, 2, 3}};
  static const uint8_t kPerm3[6][4] = {{0, 1, 2, 3}, {0, 2, 1, 3}, {1, 0, 2, 3},
                                       {1, 2, 0, 3}, {2, 0, 1, 3}, {2, 1, 0, 3}};
  uint8_t perm4[24][4];
  {
    uint8_t a[4] = {0, 1, 2, 3};
    int n = 0;
    do {
      for (int k = 0; k < 4; ++k) perm4[n][k] = a[k];
      ++n;
    } while (std::next_permutation(a, a + 4));
  }
  // Cost of element e in a group with residue masks used[]: repeated
  // residues over its fanin positions, for the best order of its fanins
  // (written to *best_p).
  auto place_cost = [&](uint32_t e, const uint32_t (&used)[4], const uint8_t** best_p) {
    const uint32_t nf = nf_of(e);
    const bool comm = gate_family(nl.type[e]) != 2;
    const uint8_t(*list)[4] = kPerm2;
    int np = 1;
    if (comm && nf == 2) {
      list = kPerm2;
      np = 2;
    } else if (comm && nf == 3) {
      list = kPerm3;
      np = 6;
    } else if (comm && nf == 4) {
      list = perm4;
      np = 24;
    }
    int best = 1 << 30;
    for (int q = 0; q < np; ++q) {
      int cost = 0;
      for (uint32_t k = 0; k < nf; ++k) cost += (used[k] >> res_in(e, list[q][k])) & 1u;
      if (cost < best) {
        best = cost;
        *best_p = list[q];
        if (cost == 0) break;
      }
    }
    return best;
  };
  std::vector<uint32_t> order, leftover;
  // Groups of G consecutive positions inside one class.  Each member is the
  // candidate (with its best fanin order) adding the fewest repeated
  // residues per fanin position to the group, none if possible; only the
  // last, partial group of a class goes to a mixed tail at the end of the
  // level.
  auto make_groups = [&](std::vector<uint32_t>& pool_in, bool tail) {
    std::vector<uint8_t> taken(pool_in.size(), 0);
    size_t left = pool_in.size(), first_free = 0;
    while (left >= G || (tail && left > 0)) {
      uint32_t used[4] = {0, 0, 0, 0};
      size_t n_grp = 0;
      while (n_grp < G && left > 0) {
        size_t best = SIZE_MAX;
        int best_cost = 1 << 30;
        const uint8_t* best_perm = kPerm2[0];
        size_t scanned = 0;
        while (first_free < pool_in.size() && taken[first_free]) ++first_free;
        for (size_t c = first_free; c < pool_in.size() && scanned < 256; ++c) {
          if (taken[c]) continue;
          ++scanned;
          const uint8_t* pp = kPerm2[0];
          const int cost = place_cost(pool_in[c], used, &pp);
          if (cost < best_cost) {
            best_cost = cost;
            best = c;
            best_perm = pp;
            if (cost == 0) break;
          }
        }
        if (best == SIZE_MAX) break;  // unreachable: left > 0 leaves a candidate
        const uint32_t e = pool_in[best];
        taken[best] = 1;
        --left;
        for (uint32_t k = 0; k < 4; ++k) perm[e][k] = best_perm[k];
        for (uint32_t k = 0; k < nf_of(e); ++k) used[k] |= 1u << res_in(e, perm[e][k]);
        order.push_back(e);
        ++n_grp;
      }
    }
    if (!tail)
      for (size_t c = 0; c < pool_in.size(); ++c)
        if (!taken[c]) leftover.push_back(pool_in[c]);
  };
  S.lvl.assign(nl.n_levels + 1, LevelDesc{0, 0, 0, 0});
  std::vector<uint64_t>& blob = S.blob;
  std::vector<uint32_t> plain, wide;
  for (uint32_t L = 1; L <= P.max_gate_level && L < nl.n_levels; ++L) {
    for (uint32_t s : release[L]) pool.release(s);
    const uint32_t lo = nl.level_off[L], hi = nl.level_off[L + 1];
    // Gates that feed a gate or a PO; a plain record holds a gate that feeds
    // gates only, with a compile-time class.
    plain.clear();
    wide.clear();
    for (uint32_t e = lo; e < hi; ++e) {
      if (!P.gate_fo[e] && !P.po_drv[e]) continue;
      if (!P.po_drv[e] && plain_class(nl.type[e], nf_of(e)) < kPlainClasses)
        plain.push_back(e);
      else
        wide.push_back(e);
    }
    order.clear();
    // Groups of G inside each class, then the classes' partial groups as a
    // mixed tail (grouped too); `key` orders the classes.
    auto part = [&](std::vector<uint32_t>& elems, const std::function<uint32_t(uint32_t)>& key) {
      std::stable_sort(elems.begin(), elems.end(), [&](uint32_t a, uint32_t b) { return key(a) < key(b); });
      leftover.clear();
      for (size_t i = 0; i < elems.size();) {
        size_t j = i;
        while (j < elems.size() && key(elems[j]) == key(elems[i])) ++j;
        std::vector<uint32_t> cls(elems.begin() + i, elems.begin() + j);
        make_groups(cls, false);
        i = j;
      }
      std::stable_sort(leftover.begin(), leftover.end(), [&](uint32_t a, uint32_t b) { return key(a) < key(b); });
      make_groups(leftover, true);
    };
    part(plain, [&](uint32_t e) { return plain_body(plain_class(nl.type[e], nf_of(e))); });
    uint32_t n_plain = (uint32_t)order.size();
    // the wide part starts on a group boundary: pad with no-op records
    const uint32_t n_pad = wide.empty() ? 0 : (G - n_plain % G) % G;
    part(wide, [&](uint32_t e) { return cls_of(e); });
    const uint32_t n_wide = (uint32_t)order.size() - n_plain;
    // Level block: plain records (8 bytes), padded to 16 bytes, then wide
    // records (16 bytes).
    while (blob.size() % 2) blob.push_back(0);
    LevelDesc& d = S.lvl[L];
    d.off16 = (uint32_t)(blob.size() / 2);
    d.n_plain = n_plain + n_pad;
    d.n_wide = n_wide;
    const size_t plain_base = blob.size();
    blob.resize(plain_base + ((size_t)d.n_plain + 1) / 2 * 2 + 2ull * n_wide, 0);
    for (uint32_t k = 0; k < n_pad; ++k) blob[plain_base + n_plain + k] = plain_rec(0, 0, 0, 0, kPNop);
    const size_t wide_base = plain_base + ((size_t)d.n_plain + 1) / 2 * 2;
    d.n16 = (uint32_t)((blob.size() - plain_base) / 2);
    S.max_block16 = std::max(S.max_block16, d.n16);
    // Positions, output slots (residue = position mod G) and records.
    std::vector<uint32_t> pos_slot[5];
    for (auto& v : pos_slot) v.assign(order.size() + n_pad, kNoSlot);
    for (uint32_t o = 0; o < order.size(); ++o) {
      const uint32_t e = order[o];
      const uint32_t pos = o < n_plain ? o : o + n_pad;
      const uint32_t nf = nf_of(e);
      uint32_t fs[4] = {0, 0, 0, 0};
      for (uint32_t k = 0; k < nf; ++k) {
        fs[k] = slot[nl.fi_idx[nl.fi_off[e] + perm[e][k]]];
        pos_slot[k][pos] = fs[k];
      }
      uint32_t out = 0;
      if (P.gate_fo[e]) {
        slot[e] = pool.alloc(pos % G);
        release[P.maxfo_level[e] + 1].push_back(slot[e]);
        out = slot[e];
        pos_slot[4][pos] = out;
      }
      const uint8_t t = nl.type[e];
      if (o < n_plain) {
        blob[plain_base + o] = plain_rec(fs[0], fs[1], fs[2], out, plain_class(t, nf));
        continue;
      }
      SweepRec r{};
      for (uint32_t k = 0; k < nf; ++k) r.fs[k] = (uint16_t)fs[k];
      uint32_t meta = (uint32_t)t & kRecTypeMask;
      meta |= ((nf ? nf - 1 : 0) & 3u) << kRecNfShift;
      meta |= gate_class(t, nf) << kRecClassShift;
      if (t == G_OR || t == G_NOR) meta |= kRecIi;
      if (t == G_INV || t == G_OR || t == G_NAND || t == G_XNOR) meta |= kRecIo;
      if (P.po_drv[e]) meta |= kRecPo;
      if (P.gate_fo[e]) {
        meta |= kRecHasSlot;
        r.slot = (uint16_t)out;
      }
      r.meta = (uint16_t)meta;
      r.elem = e;
      std::memcpy(&blob[wide_base + 2ull * (o - n_plain)], &r, sizeof r);
    }
    // Bank-conflict accounting per aligned group of G positions.
    const uint32_t n_pos = (uint32_t)order.size() + n_pad;
    for (uint32_t g0 = 0; g0 < n_pos; g0 += G) {
      const uint32_t g1 = std::min<uint32_t>(g0 + G, n_pos);
      for (uint32_t k = 0; k < 5; ++k) {
        uint32_t seen = 0, any = 0;
        bool conflict = false;
        for (uint32_t o = g0; o < g1; ++o) {
          const uint32_t sl = pos_slot[k][o];
          if (sl == kNoSlot) continue;
          any = 1;
          conflict |= (seen >> (sl % G)) & 1u;
          seen |= 1u << (sl % G);
        }
        S.access_groups += any;
        S.conflict_groups += conflict;
      }
    }
  }
  S.max_live = pool.next_block * G;
  if (S.max_live > kMaxSlots) {
    S.blob.clear();
    return;
  }
  // Live-in sets as (element, slot) pairs.
  std::vector<uint32_t> cnt(nl.n_levels + 2, 0);
  for (uint32_t e = 0; e < N; ++e)
    if (slot[e] != kNoSlot)
      for (uint32_t l = nl.level[e] + 1; l <= P.maxfo_level[e]; ++l) cnt[l]++;
  S.li_off.assign(nl.n_levels + 1, 0);
  for (uint32_t l = 0; l < nl.n_levels; ++l) S.li_off[l + 1] = S.li_off[l] + cnt[l];
  S.li.assign(2ull * S.li_off[nl.n_levels], 0);
  std::vector<uint32_t> fill(S.li_off.begin(), S.li_off.end() - 1);
  for (uint32_t e = 0; e < N; ++e)
    if (slot[e] != kNoSlot)
      for (uint32_t l = nl.level[e] + 1; l <= P.maxfo_level[e]; ++l) {
        const uint32_t i = fill[l]++;
        S.li[2 * i] = e;
        S.li[2 * i + 1] = slot[e];
      }
}

}  // namespace fsimb
