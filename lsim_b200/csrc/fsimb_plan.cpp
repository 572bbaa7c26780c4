// Netlist + fault list -> device plan (see fsimb_plan.h).
#include "fsimb_plan.h"

#include <algorithm>

namespace fsimb {

void build_plan(const Netlist& nl, const std::vector<Fault>& faults, Plan& P) {
  P = Plan();
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
  std::vector<uint8_t> po_drv(N, 0), gate_fo(N, 0), mux_below(N, 0);
  P.maxfo_level.assign(N, 0);
  for (uint32_t e = 0; e < N; ++e) {
    for (uint32_t k = nl.fo_off[e]; k < nl.fo_off[e + 1]; ++k) {
      uint32_t c = nl.fo_idx[k];
      if (nl.type[c] == G_PO) {
        po_drv[e] = 1;
      } else {
        gate_fo[e] = 1;
        P.maxfo_level[e] = std::max(P.maxfo_level[e], nl.level[c]);
      }
    }
    P.has_mux |= nl.type[e] == G_MUX;
  }
  for (int64_t e = (int64_t)N - 1; e >= 0; --e) {
    uint8_t hb = 0;
    for (uint32_t k = nl.fo_off[e]; k < nl.fo_off[e + 1]; ++k) {
      uint32_t c = nl.fo_idx[k];
      hb |= (nl.type[c] == G_MUX) | mux_below[c];
    }
    mux_below[e] = hb;
  }

  // Shared-memory slots: interval allocation over live ranges
  // [level(e), highest consumer level].  Intervals sharing a slot never
  // overlap, so a slot is rewritten only after its last reader's level.
  std::vector<uint32_t> slot(N, kNoSlot);
  {
    std::vector<std::vector<uint32_t>> release(nl.n_levels + 1);
    std::vector<uint32_t> free_slots;
    uint32_t next = 0, live = 0;
    for (uint32_t l = 0; l < nl.n_levels; ++l) {
      for (uint32_t s : release[l]) {
        free_slots.push_back(s);
        --live;
      }
      for (uint32_t e = nl.level_off[l]; e < nl.level_off[l + 1]; ++e) {
        if (!gate_fo[e]) continue;
        uint32_t s;
        if (!free_slots.empty()) {
          s = free_slots.back();
          free_slots.pop_back();
        } else {
          s = next++;
        }
        slot[e] = s;
        ++live;
        release[P.maxfo_level[e] + 1].push_back(s);
      }
      P.max_live = std::max(P.max_live, live);
    }
    P.max_live = std::max(P.max_live, next);
  }

  // Sweep records.
  P.fslot.assign((size_t)N * 4, 0);
  P.meta.assign(N, 0);
  for (uint32_t e = 0; e < N; ++e) {
    const uint8_t t = nl.type[e];
    uint32_t nf = nl.fanin_count(e);
    // INV, CLKBUF and PO read their first input only (fsim/simulation.cpp:979-983,
    // 1062-1067, 1074-1077).
    if (t == G_INV || t == G_CLKBUF || t == G_PO) nf = std::min<uint32_t>(nf, 1);
    for (uint32_t k = 0; k < nf && k < 4; ++k) P.fslot[(size_t)e * 4 + k] = slot[nl.fi_idx[nl.fi_off[e] + k]];
    uint32_t m = (slot[e] == kNoSlot ? kNoSlot : slot[e]) & kMetaSlotMask;
    if (slot[e] != kNoSlot) m |= kMetaHasSlot;
    if (po_drv[e]) m |= kMetaPo;
    m |= ((nf ? nf - 1 : 0) & 3u) << kMetaNfShift;
    m |= ((uint32_t)t & 15u) << kMetaTypeShift;
    P.meta[e] = m;
  }

  // Live-in sets: elements whose value a sweep starting at level L reads
  // before computing it (level(e) < L <= highest consumer level).
  {
    std::vector<uint32_t> cnt(nl.n_levels + 2, 0);
    for (uint32_t e = 0; e < N; ++e)
      if (slot[e] != kNoSlot)
        for (uint32_t l = nl.level[e] + 1; l <= P.maxfo_level[e]; ++l) cnt[l]++;
    P.li_off.assign(nl.n_levels + 1, 0);
    for (uint32_t l = 0; l < nl.n_levels; ++l) P.li_off[l + 1] = P.li_off[l] + cnt[l];
    P.li_elem.assign(P.li_off[nl.n_levels], 0);
    std::vector<uint32_t> fill(P.li_off.begin(), P.li_off.end() - 1);
    for (uint32_t e = 0; e < N; ++e)
      if (slot[e] != kNoSlot)
        for (uint32_t l = nl.level[e] + 1; l <= P.maxfo_level[e]; ++l) P.li_elem[fill[l]++] = e;
  }

  // FFR roots.
  std::vector<uint32_t> root(N);
  for (int64_t e = (int64_t)N - 1; e >= 0; --e) {
    uint32_t fo = nl.fo_off[e + 1] - nl.fo_off[e];
    if (nl.type[e] == G_PO || fo != 1)
      root[e] = (uint32_t)e;
    else
      root[e] = root[nl.fo_idx[nl.fo_off[e]]];
  }

  // Classify faults.
  std::vector<uint32_t> root_id(N, UINT32_MAX);
  std::vector<std::vector<uint32_t>> root_faults;
  std::vector<uint32_t> root_elem;
  for (uint32_t f = 0; f < faults.size(); ++f) {
    const Fault& ft = faults[f];
    const uint32_t x = ft.site;
    bool exact = ft.pin == 0 ? mux_below[x] : (nl.type[x] == G_MUX || mux_below[x]);
    if (exact) continue;
    uint32_t r = root[x];
    if (root_id[r] == UINT32_MAX) {
      root_id[r] = (uint32_t)root_elem.size();
      root_elem.push_back(r);
      root_faults.emplace_back();
    }
    root_faults[root_id[r]].push_back(f);
  }
  // Members of the FFRs that carry traced faults, descending (consumer first).
  std::vector<std::vector<uint32_t>> root_members(root_elem.size());
  for (int64_t e = (int64_t)N - 1; e >= 0; --e) {
    uint32_t r = root[e];
    if (r != (uint32_t)e && root_id[r] != UINT32_MAX) root_members[root_id[r]].push_back((uint32_t)e);
  }
  // Order roots by level so neighbouring warps touch neighbouring data.
  std::vector<uint32_t> rorder(root_elem.size());
  for (uint32_t i = 0; i < rorder.size(); ++i) rorder[i] = i;
  std::sort(rorder.begin(), rorder.end(), [&](uint32_t a, uint32_t b) { return root_elem[a] < root_elem[b]; });
  for (uint32_t ri : rorder) {
    const uint32_t r = root_elem[ri];
    RootRec rr{};
    rr.root = r;
    if (nl.type[r] == G_PO || po_drv[r])
      rr.obs = kObsOne;
    else if (!gate_fo[r])
      rr.obs = kObsZero;
    else {
      rr.obs = (uint32_t)P.sweeps.size();
      P.sweeps.push_back(InjRec{r, 0, 0, 0});
      P.sweep_root.push_back((uint32_t)P.roots.size());
    }
    rr.mem_begin = (uint32_t)P.members.size();
    for (uint32_t e : root_members[ri]) {
      uint32_t k = nl.fo_off[e];
      P.members.push_back(MemberRec{e, nl.fo_idx[k], nl.fo_pin[k], 0});
    }
    rr.mem_end = (uint32_t)P.members.size();
    rr.flt_begin = (uint32_t)P.traced.size();
    for (uint32_t f : root_faults[ri])
      P.traced.push_back(TracedRec{f, faults[f].site, faults[f].pin, faults[f].value});
    rr.flt_end = (uint32_t)P.traced.size();
    P.roots.push_back(rr);
  }
  P.n_stem_sweeps = (uint32_t)P.sweeps.size();
  for (uint32_t f = 0; f < faults.size(); ++f) {
    const Fault& ft = faults[f];
    const uint32_t x = ft.site;
    bool exact = ft.pin == 0 ? mux_below[x] : (nl.type[x] == G_MUX || mux_below[x]);
    if (!exact) continue;
    P.sweeps.push_back(InjRec{x, ft.pin, 1, ft.value});
    P.exact_fault.push_back(f);
  }
  // Algorithmic bytes of one gate-word evaluation: its fanin words read and
  // its output word written, 8 * (fanin + 1).
  P.nfp_prefix.assign(N + 1, 0);
  for (uint32_t e = 0; e < N; ++e) {
    uint32_t nf = ((P.meta[e] >> kMetaNfShift) & 3u) + 1u;
    if (e < P.n_pi) nf = 0;
    P.nfp_prefix[e + 1] = P.nfp_prefix[e] + 8ull * (nf + 1);
  }
  const uint32_t gates_end = nl.level_off[std::min(P.max_gate_level + 1, nl.n_levels)];
  for (auto& s : P.sweeps) {
    uint32_t L0 = nl.level[s.elem] + 1;
    if (L0 <= P.max_gate_level) {
      P.dense_sweep_gates += gates_end - nl.level_off[L0];
      P.dense_sweep_bytes += P.nfp_prefix[gates_end] - P.nfp_prefix[nl.level_off[L0]];
    }
  }
}

}  // namespace fsimb
