// Synthetic circuit, pattern and fault-list generators (see fsimb_gen.h).
#include "fsimb_gen.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <numeric>

namespace fsimb {

namespace {

// xoshiro256** seeded through splitmix64: deterministic on every platform.
struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) {
      x += 0x9E3779B97F4A7C15ull;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      s[i] = z ^ (z >> 31);
    }
  }
  static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
  uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  uint64_t below(uint64_t n) { return n ? next() % n : 0; }
  double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

void append_u64(std::string& s, uint64_t v) {
  char buf[24];
  int n = snprintf(buf, sizeof buf, "%llu", (unsigned long long)v);
  s.append(buf, n);
}

}  // namespace

std::string generate_ckt(const GenConfig& cfg) {
  Rng rng(cfg.seed * 0x100000001B3ull + 0x5151);
  const uint32_t nPI = cfg.n_pi, nPO = cfg.n_po, nG = cfg.n_gates;
  const uint32_t L = std::max<uint32_t>(1, std::min(cfg.n_levels, std::max<uint32_t>(1, nG)));
  // Node ids: PIs [0, nPI), gates nPI + g in creation order.
  const uint32_t nodes = nPI + nG;
  std::vector<uint32_t> lvl_begin(L + 2, 0);
  lvl_begin[0] = 0;
  lvl_begin[1] = nPI;
  for (uint32_t l = 1; l <= L; ++l) {
    uint32_t sz = nG / L + (l - 1 < nG % L ? 1 : 0);
    lvl_begin[l + 1] = lvl_begin[l] + sz;
  }
  std::vector<uint32_t> fo(nodes, 0), target(nodes, 0);
  const bool hub_mode = cfg.hub_frac > 0.0;
  if (hub_mode) {
    for (uint32_t v = 0; v < nodes; ++v) {
      if (rng.unit() < cfg.hub_frac)
        target[v] = cfg.hub_fo_min + (uint32_t)rng.below(cfg.hub_fo_max - cfg.hub_fo_min + 1);
      else
        target[v] = cfg.fo_min + (uint32_t)rng.below(cfg.fo_max - cfg.fo_min + 1);
    }
  }
  // Urn per level: preferential attachment (weight 1 + fanout) or, in hub
  // mode, one token per unit of remaining fanout target.
  std::vector<std::vector<uint32_t>> urn(L + 1);
  std::vector<std::vector<uint32_t>> unused(L + 1);
  std::vector<size_t> unused_head(L + 1, 0);
  auto add_node = [&](uint32_t v, uint32_t l) {
    if (hub_mode) {
      for (uint32_t k = 0; k < target[v]; ++k) urn[l].push_back(v);
    } else {
      urn[l].push_back(v);
    }
    unused[l].push_back(v);
  };
  for (uint32_t i = 0; i < nPI; ++i) add_node(i, 0);
  // Shuffle the unused lists lazily by picking random entries.
  auto pick_unused = [&](uint32_t l) -> int64_t {
    auto& u = unused[l];
    while (!u.empty()) {
      size_t i = (size_t)rng.below(u.size());
      uint32_t v = u[i];
      u[i] = u.back();
      u.pop_back();
      if (fo[v] == 0) return v;
    }
    return -1;
  };
  auto pick_urn = [&](uint32_t lo, uint32_t hi) -> int64_t {
    size_t total = 0;
    for (uint32_t l = lo; l <= hi; ++l) total += urn[l].size();
    if (total == 0) {
      size_t span = lvl_begin[hi + 1] - lvl_begin[lo];
      if (span == 0) return -1;
      return lvl_begin[lo] + (uint32_t)rng.below(span);
    }
    size_t r = (size_t)rng.below(total);
    for (uint32_t l = lo; l <= hi; ++l) {
      if (r < urn[l].size()) {
        uint32_t v = urn[l][r];
        if (hub_mode) {
          urn[l][r] = urn[l].back();
          urn[l].pop_back();
        } else {
          urn[l].push_back(v);
        }
        return v;
      }
      r -= urn[l].size();
    }
    return -1;
  };

  std::vector<uint8_t> gtype(nG);
  std::vector<uint32_t> fin_off(nG + 1, 0), fin;
  fin.reserve((size_t)nG * 3);
  std::vector<uint8_t> allowed;
  for (uint8_t t = 0; t <= 8; ++t)
    if (cfg.type_mask & (1u << t)) allowed.push_back(t);
  if (allowed.empty()) allowed.push_back(G_AND);

  for (uint32_t l = 1; l <= L; ++l) {
    const uint32_t lo = (l > cfg.window) ? l - cfg.window : 0;
    for (uint32_t v = lvl_begin[l]; v < lvl_begin[l + 1]; ++v) {
      const uint32_t g = v - nPI;
      uint8_t t = allowed[rng.below(allowed.size())];
      uint32_t k;
      if (t == G_INV || t == G_CLKBUF)
        k = 1;
      else if (t == G_MUX)
        k = 3;
      else
        k = (rng.unit() < cfg.p_fanin3) ? 3 : 2;
      gtype[g] = t;
      uint32_t chosen[4];
      uint32_t nc = 0;
      int64_t s = pick_unused(l - 1);
      if (s < 0) s = pick_urn(l - 1, l - 1);
      chosen[nc++] = (uint32_t)s;
      for (uint32_t j = 1; j < k; ++j) {
        int64_t c = -1;
        for (int attempt = 0; attempt < 16 && c < 0; ++attempt) {
          int64_t cand = -1;
          if (rng.unit() < cfg.p_unused) {
            for (uint32_t ll = lo; ll < l && cand < 0; ++ll) cand = pick_unused(ll);
          }
          if (cand < 0) cand = pick_urn(lo, l - 1);
          bool dup = false;
          for (uint32_t q = 0; q < nc; ++q) dup |= (chosen[q] == (uint32_t)cand);
          if (!dup) c = cand;
        }
        if (c < 0) {  // deterministic fallback: first distinct node of the window
          for (uint32_t x = lvl_begin[lo]; x < lvl_begin[l] && c < 0; ++x) {
            bool dup = false;
            for (uint32_t q = 0; q < nc; ++q) dup |= (chosen[q] == x);
            if (!dup) c = x;
          }
        }
        if (c < 0) break;
        chosen[nc++] = (uint32_t)c;
      }
      if (t == G_MUX && nc < 3) {
        gtype[g] = G_AND;
      }
      for (uint32_t q = 0; q < nc; ++q) {
        fin.push_back(chosen[q]);
        fo[chosen[q]]++;
      }
      fin_off[g + 1] = (uint32_t)fin.size();
      add_node(v, l);
    }
  }

  // PO drivers: sink gates from the top level down, then other top gates.
  std::vector<uint32_t> po_drv;
  po_drv.reserve(nPO);
  std::vector<uint8_t> taken(nodes, 0);
  for (uint32_t l = L; l >= 1 && po_drv.size() < nPO; --l) {
    std::vector<uint32_t> sinks;
    for (uint32_t v = lvl_begin[l]; v < lvl_begin[l + 1]; ++v)
      if (fo[v] == 0) sinks.push_back(v);
    for (size_t i = sinks.size(); i > 1; --i) std::swap(sinks[i - 1], sinks[rng.below(i)]);
    for (uint32_t v : sinks) {
      if (po_drv.size() >= nPO) break;
      po_drv.push_back(v);
      taken[v] = 1;
    }
    if (l == 1) break;
  }
  for (uint32_t l = L; l >= 1 && po_drv.size() < nPO; --l) {
    for (uint32_t v = lvl_begin[l]; v < lvl_begin[l + 1] && po_drv.size() < nPO; ++v) {
      if (!taken[v]) {
        po_drv.push_back(v);
        taken[v] = 1;
      }
    }
    if (l == 1) break;
  }
  for (uint32_t i = 0; po_drv.size() < nPO; ++i) po_drv.push_back(i % std::max<uint32_t>(1, nPI));
  for (size_t i = po_drv.size(); i > 1; --i) std::swap(po_drv[i - 1], po_drv[rng.below(i)]);

  // File ids.
  std::vector<uint32_t> gate_fid(nG);
  std::iota(gate_fid.begin(), gate_fid.end(), nPI + nPO);
  if (cfg.shuffle_ids)
    for (size_t i = gate_fid.size(); i > 1; --i) std::swap(gate_fid[i - 1], gate_fid[rng.below(i)]);
  auto fid = [&](uint32_t node) { return node < nPI ? node : gate_fid[node - nPI]; };
  const uint32_t Nf = nPI + nPO + nG;
  // Sink lists per source file id.
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> sinks(Nf);
  for (uint32_t g = 0; g < nG; ++g) {
    for (uint32_t k = fin_off[g]; k < fin_off[g + 1]; ++k) {
      uint32_t pin = k - fin_off[g] + 1;
      if (gtype[g] == G_MUX && pin == 3) pin = 5;
      sinks[fid(fin[k])].push_back({gate_fid[g], pin});
    }
  }
  for (uint32_t i = 0; i < nPO; ++i) sinks[fid(po_drv[i])].push_back({nPI + i, 1});
  uint64_t n_wires = 0;
  for (auto& s : sinks) n_wires += !s.empty();
  std::vector<uint8_t> ftype(Nf, 0);
  for (uint32_t g = 0; g < nG; ++g) ftype[gate_fid[g]] = gtype[g];

  std::string out;
  out.reserve((size_t)nG * 40 + 64);
  append_u64(out, nPI);
  out += '\n';
  append_u64(out, nPO);
  out += '\n';
  append_u64(out, nG);
  out += '\n';
  append_u64(out, n_wires);
  out += '\n';
  for (uint32_t f = 0; f < Nf; ++f) {
    if (sinks[f].empty()) continue;
    append_u64(out, f);
    out += " 0 ";
    append_u64(out, sinks[f].size());
    for (auto& pr : sinks[f]) {
      out += ' ';
      append_u64(out, pr.first);
      out += ' ';
      append_u64(out, pr.second);
    }
    out += '\n';
  }
  for (uint32_t f = nPI + nPO; f < Nf; ++f) {
    append_u64(out, ftype[f]);
    out += (f + 1 < Nf) ? ' ' : '\n';
  }
  if (nG == 0) out += '\n';
  return out;
}

void generate_patterns(const PatternConfig& cfg, uint64_t n_pi, Patterns& out) {
  Rng rng(cfg.seed * 0x9E3779B97F4A7C15ull + 0x7A7A);
  out = Patterns();
  out.P = cfg.n_patterns;
  out.W = (out.P + 63) / 64;
  out.words.assign(out.W * n_pi, 0);
  std::vector<uint8_t> biased(n_pi, 0);
  for (uint64_t b = 0; b < n_pi; ++b) biased[b] = rng.unit() < cfg.biased_pi_frac;
  // Threshold for P(bit = 1) = p_one_biased using 16-bit uniforms.
  const uint32_t thr = (uint32_t)std::lround(cfg.p_one_biased * 65536.0);
  for (uint64_t w = 0; w < out.W; ++w) {
    const uint32_t bits = out.bits(w);
    const uint64_t mask = bits == 64 ? ~0ull : ((1ull << bits) - 1);
    for (uint64_t b = 0; b < n_pi; ++b) {
      uint64_t v;
      if (!biased[b]) {
        v = rng.next();
      } else {
        v = 0;
        for (int q = 0; q < 16; ++q) {
          uint64_t r = rng.next();
          for (int h = 0; h < 4; ++h) {
            uint64_t bit = ((r >> (16 * h)) & 0xFFFF) < thr;
            v |= bit << (q * 4 + h);
          }
        }
      }
      out.words[w * n_pi + b] = v & mask;
    }
  }
}

std::string write_ptn(const Patterns& p, uint64_t n_pi) {
  std::string s;
  s.reserve(p.words.size() * 21 + 32);
  append_u64(s, p.P);
  s += '\n';
  for (uint64_t w = 0; w < p.W; ++w) {
    for (uint64_t b = 0; b < n_pi; ++b) {
      append_u64(s, p.words[w * n_pi + b]);
      s += ' ';
    }
    s += '\n';
  }
  return s;
}

namespace {

struct UF {
  std::vector<uint32_t> p;
  explicit UF(size_t n) : p(n) { std::iota(p.begin(), p.end(), 0u); }
  uint32_t find(uint32_t x) {
    while (p[x] != x) {
      p[x] = p[p[x]];
      x = p[x];
    }
    return x;
  }
  void unite(uint32_t a, uint32_t b) {
    a = find(a);
    b = find(b);
    if (a != b) p[std::max(a, b)] = std::min(a, b);
  }
};

}  // namespace

void build_fault_list(const Netlist& nl, FaultListKind kind, std::vector<Fault>& out) {
  out.clear();
  const uint32_t N = nl.N;
  const uint32_t g0 = (uint32_t)nl.n_pi, g1 = (uint32_t)(nl.n_pi + nl.n_gates);
  // Gates by file id, SA0 then SA1.
  std::vector<uint32_t> gates_by_fid;
  gates_by_fid.reserve(nl.n_gates);
  for (uint64_t f = nl.n_pi + nl.n_po; f < N; ++f) gates_by_fid.push_back((uint32_t)nl.tpg[f]);
  if (kind == FL_OUTPUTS || kind == FL_OUTPUTS_AND_PINS) {
    for (uint32_t t : gates_by_fid) {
      out.push_back(Fault{t, 0, 0});
      out.push_back(Fault{t, 0, 1});
      if (kind == FL_OUTPUTS_AND_PINS) {
        for (uint32_t k = 0; k < nl.fanin_count(t); ++k) {
          out.push_back(Fault{t, (uint8_t)(k + 1), 0});
          out.push_back(Fault{t, (uint8_t)(k + 1), 1});
        }
      }
    }
    return;
  }
  // Equivalence collapsing over lines: a stem line per element, a branch line
  // per consumer pin whose driver fans out more than once.
  const uint32_t E = nl.fi_off[N];
  auto fo_count = [&](uint32_t d) { return nl.fo_off[d + 1] - nl.fo_off[d]; };
  auto pin_line = [&](uint32_t h, uint32_t k) -> uint32_t {
    uint32_t d = nl.fi_idx[nl.fi_off[h] + k];
    return fo_count(d) == 1 ? d : N + nl.fi_off[h] + k;
  };
  UF uf((size_t)(N + E) * 2);
  for (uint32_t h = g0; h < N; ++h) {
    const uint32_t o = h;
    const uint8_t t = nl.type[h];
    const uint32_t nin = nl.fanin_count(h);
    for (uint32_t k = 0; k < nin; ++k) {
      const uint32_t i = pin_line(h, k);
      switch (t) {
        case G_AND: uf.unite(2 * i + 0, 2 * o + 0); break;
        case G_NAND: uf.unite(2 * i + 0, 2 * o + 1); break;
        case G_OR: uf.unite(2 * i + 1, 2 * o + 1); break;
        case G_NOR: uf.unite(2 * i + 1, 2 * o + 0); break;
        case G_INV:
          if (k == 0) {
            uf.unite(2 * i + 0, 2 * o + 1);
            uf.unite(2 * i + 1, 2 * o + 0);
          }
          break;
        case G_CLKBUF:
        case G_PO:
          if (k == 0) {
            uf.unite(2 * i + 0, 2 * o + 0);
            uf.unite(2 * i + 1, 2 * o + 1);
          }
          break;
        default: break;  // XOR, XNOR, MUX: no equivalences
      }
    }
  }
  // Universe: inner-gate outputs and inner-gate input pins.  Each member is
  // written as a concrete fault; a fanout-free pin becomes its driver's
  // output fault (same line).
  struct Member {
    uint32_t cls;
    Fault f;
  };
  std::vector<Member> members;
  members.reserve((size_t)(g1 - g0) * 8);
  for (uint32_t h = g0; h < g1; ++h) {
    for (uint8_t v = 0; v < 2; ++v) members.push_back({uf.find(2 * h + v), Fault{h, 0, v}});
    for (uint32_t k = 0; k < nl.fanin_count(h); ++k) {
      uint32_t d = nl.fi_idx[nl.fi_off[h] + k];
      uint32_t line = pin_line(h, k);
      for (uint8_t v = 0; v < 2; ++v) {
        Fault f = (line == d) ? Fault{d, 0, v} : Fault{h, (uint8_t)(k + 1), v};
        members.push_back({uf.find(2 * line + v), f});
      }
    }
  }
  // Representative: output faults first, then lowest (site, pin).
  auto key = [](const Fault& f) {
    return ((uint64_t)(f.pin != 0) << 40) | ((uint64_t)f.site << 8) | f.pin;
  };
  std::vector<uint64_t> best((size_t)(N + E) * 2, UINT64_MAX);
  std::vector<Fault> best_f((size_t)(N + E) * 2);
  for (auto& m : members) {
    uint64_t kk = key(m.f) * 2 + m.f.value;
    if (kk < best[m.cls]) {
      best[m.cls] = kk;
      best_f[m.cls] = m.f;
    }
  }
  for (size_t c = 0; c < best.size(); ++c)
    if (best[c] != UINT64_MAX) out.push_back(best_f[c]);
  std::sort(out.begin(), out.end(), [](const Fault& a, const Fault& b) {
    if (a.site != b.site) return a.site < b.site;
    if (a.pin != b.pin) return a.pin < b.pin;
    return a.value < b.value;
  });
}

std::string write_flst(const Netlist& nl, const std::vector<Fault>& faults, bool force_pins) {
  bool pins = force_pins;
  for (auto& f : faults) pins |= f.pin != 0;
  std::vector<uint32_t> order(nl.N);
  for (uint32_t f = 0; f < nl.N; ++f) order[nl.tpg[f]] = f;
  std::string s;
  s.reserve(faults.size() * 16 + 32);
  if (pins) s += "@pins\n";
  append_u64(s, faults.size());
  s += '\n';
  for (auto& f : faults) {
    append_u64(s, order[f.site]);
    s += ' ';
    append_u64(s, f.value);
    if (pins) {
      s += ' ';
      append_u64(s, f.pin);
    }
    s += '\n';
  }
  return s;
}

}  // namespace fsimb
