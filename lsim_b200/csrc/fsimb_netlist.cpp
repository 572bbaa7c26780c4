// Readers and levelizer.  The element ordering, fanin order, level numbering,
// fault and pattern conventions restate fsim/simulation.cpp:37-63 and
// 664-976 exactly; see fsimb_netlist.h for the per-step citations.
//
// Inputs on which the reference reader has undefined behaviour are rejected:
//   * a pin number outside 1..5, or more than four inputs on one element
//     (fsim/simulation.cpp:679 sizes the pin table to 5 slots);
//   * a wire that drives a PI or starts at a PO (breaks the PI seeding and
//     the PO re-append at fsim/simulation.cpp:728-751);
//   * elements not reachable from the PIs (no fanin, or a cycle): the
//     reference then indexes past `order` (fsim/simulation.cpp:797-819);
//   * a PO without a driver, or a MUX with fewer than three inputs
//     (fsim/simulation.cpp:1054-1056, 1072-1076 read missing inputs);
// Pin-slot gaps and repeated pins, which the reference accepts, are kept
// with the reference's meaning (fanin = slots 1..count); when they leave the
// element order not level-sorted, the schedule levels differ from the
// reference's levels (finalize_netlist) and the results do not.
// A PI that directly drives a PO is accepted and the PO copies the PI; the
// reference writes past its gate array in that case (fsim/simulation.cpp:856-861).
#include "fsimb_netlist.h"

#include <algorithm>
#include <cstring>

namespace fsimb {

namespace {

inline bool is_ws(char c) {
  return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\f' || c == '\v';
}

struct Tok {
  const char* p;
  const char* e;
  const char* what;

  void skip_ws() {
    while (p < e && is_ws(*p)) ++p;
  }
  bool at_end() {
    skip_ws();
    return p >= e;
  }
  [[noreturn]] void fail(const std::string& m) { throw ParseError{std::string(what) + ": " + m}; }
  uint64_t u64(const char* field) {
    skip_ws();
    if (p >= e) fail(std::string("unexpected end of input reading ") + field);
    if (*p < '0' || *p > '9') {
      fail(std::string("expected an unsigned integer for ") + field + ", got '" +
           std::string(p, std::min<size_t>(16, e - p)) + "'");
    }
    // 19 digits always fit in 64 bits; only a 20th needs the overflow check
    uint64_t v = 0;
    int n = 0;
    while (p < e && (unsigned)(*p - '0') < 10u && n < 19) {
      v = v * 10 + (uint64_t)(*p - '0');
      ++p;
      ++n;
    }
    if (p < e && (unsigned)(*p - '0') < 10u) {
      const uint64_t d = (uint64_t)(*p - '0');
      if (v > (UINT64_MAX - d) / 10) fail(std::string("integer overflow in ") + field);
      v = v * 10 + d;
      ++p;
      if (p < e && (unsigned)(*p - '0') < 10u) fail(std::string("integer overflow in ") + field);
    }
    if (p < e && !is_ws(*p)) fail(std::string("malformed integer in ") + field);
    return v;
  }
  bool peek_word(const char* w) {
    skip_ws();
    size_t n = strlen(w);
    if ((size_t)(e - p) >= n && memcmp(p, w, n) == 0) {
      p += n;
      return true;
    }
    return false;
  }
};

}  // namespace

void finalize_netlist(Netlist& nl) {
  const uint32_t N = nl.N;
  const uint32_t g0 = (uint32_t)nl.n_pi, g1 = (uint32_t)(nl.n_pi + nl.n_gates);
  // Levels (fsim/simulation.cpp:882-916): PIs 0, gates 1 + max fanin, POs
  // max+1.  `running` also keeps each gate at or above the gate before it in
  // element order: the schedule's level, equal to the reference's whenever
  // the element order is level-sorted.
  auto levelize = [&](bool running, std::vector<uint32_t>& level) {
    level.assign(N, 0);
    uint32_t max_level = 0;
    for (uint32_t t = g0; t < g1; ++t) {
      uint32_t lv = running && t > g0 ? level[t - 1] : 0;
      for (uint32_t k = nl.fi_off[t]; k < nl.fi_off[t + 1]; ++k)
        lv = std::max(lv, level[nl.fi_idx[k]] + 1);
      level[t] = lv;
      max_level = std::max(max_level, lv);
    }
    for (uint32_t t = g1; t < N; ++t) level[t] = max_level + 1;
    return max_level + 2;
  };
  auto histogram = [&](const std::vector<uint32_t>& level, uint32_t n_levels) {
    std::vector<uint64_t> h(n_levels, 0);
    for (uint32_t t = 0; t < N; ++t) h[level[t]]++;
    return h;
  };
  nl.n_levels = levelize(false, nl.level);
  nl.per_level = histogram(nl.level, nl.n_levels);
  nl.ref_level.clear();
  nl.ref_per_level.clear();
  bool sorted = true;
  for (uint32_t t = 1; t < N && sorted; ++t) sorted = nl.level[t] >= nl.level[t - 1];
  if (!sorted) {
    // Pin-slot gaps or repeated pins drop an edge from a gate's fanin while
    // the edge still orders the gate (fsim/simulation.cpp:697-703, 851-877):
    // keep the reference's levels for the level queries and schedule by the
    // running levels, which every fanin precedes.
    nl.ref_level.swap(nl.level);
    nl.ref_per_level.swap(nl.per_level);
    nl.n_levels = levelize(true, nl.level);
    nl.per_level = histogram(nl.level, nl.n_levels);
  }
  nl.level_off.assign(nl.n_levels + 1, 0);
  {
    uint32_t acc = 0;
    for (uint32_t l = 0; l < nl.n_levels; ++l) {
      nl.level_off[l] = acc;
      acc += (uint32_t)nl.per_level[l];
    }
    nl.level_off[nl.n_levels] = acc;
  }
  // Fanout CSR, consumers ascending.
  const uint32_t E = nl.fi_off[N];
  nl.fo_off.assign(N + 1, 0);
  for (uint32_t k = 0; k < E; ++k) nl.fo_off[nl.fi_idx[k] + 1]++;
  for (uint32_t t = 0; t < N; ++t) nl.fo_off[t + 1] += nl.fo_off[t];
  nl.fo_idx.assign(E, 0);
  nl.fo_pin.assign(E, 0);
  std::vector<uint32_t> fill(nl.fo_off.begin(), nl.fo_off.end() - 1);
  for (uint32_t t = 0; t < N; ++t) {
    for (uint32_t k = nl.fi_off[t]; k < nl.fi_off[t + 1]; ++k) {
      uint32_t d = nl.fi_idx[k];
      uint32_t pos = fill[d]++;
      nl.fo_idx[pos] = t;
      nl.fo_pin[pos] = (uint8_t)(k - nl.fi_off[t]);
    }
  }
}

void parse_ckt(const char* text, size_t len, Netlist& nl) {
  Tok tk{text, text + len, "ckt"};
  nl = Netlist();
  nl.n_pi = tk.u64("nPI");
  nl.n_po = tk.u64("nPO");
  nl.n_gates = tk.u64("nGates");
  nl.n_wires = tk.u64("nWires");
  const uint64_t N64 = nl.n_pi + nl.n_po + nl.n_gates;
  if (nl.n_pi == 0) tk.fail("a circuit needs at least one PI");
  if (N64 >= (1ull << 31) || nl.n_pi >= (1ull << 31) || nl.n_po >= (1ull << 31) ||
      nl.n_gates >= (1ull << 31))
    tk.fail("too many elements");
  if (nl.n_wires > len) tk.fail("wire count exceeds the input size");
  const uint32_t N = (uint32_t)N64;
  const uint32_t nPI = (uint32_t)nl.n_pi, nPO = (uint32_t)nl.n_po;
  nl.N = N;

  // Pin-slot table (fsim/simulation.cpp:673-711): slot[0] = count, slots 1..4.
  std::vector<uint32_t> slot((size_t)N * 5, 0);
  std::vector<uint32_t> indeg(N, 0);
  std::vector<uint32_t> e_src, e_dst;
  e_src.reserve((size_t)N * 3);
  e_dst.reserve((size_t)N * 3);
  for (uint64_t i = 0; i < nl.n_wires; ++i) {
    uint64_t src = tk.u64("wire source");
    (void)tk.u64("wire output pin");
    uint64_t k = tk.u64("wire fanout count");
    if (src >= N) tk.fail("wire source " + std::to_string(src) + " out of range");
    if (src >= nPI && src < (uint64_t)nPI + nPO)
      tk.fail("wire source " + std::to_string(src) + " is a PO");
    if (k > len) tk.fail("wire fanout count exceeds the input size");
    for (uint64_t j = 0; j < k; ++j) {
      uint64_t dst = tk.u64("wire sink");
      uint64_t pin = tk.u64("wire sink pin");
      if (dst >= N) tk.fail("wire sink " + std::to_string(dst) + " out of range");
      if (dst < nPI) tk.fail("wire sink " + std::to_string(dst) + " is a PI");
      if (pin < 1 || pin > 5) tk.fail("pin " + std::to_string(pin) + " outside 1..5");
      if (pin == 5) pin = 3;  // MUX select (fsim/simulation.cpp:703)
      uint32_t* s = &slot[(size_t)dst * 5];
      if (s[0] >= 4) tk.fail("element " + std::to_string(dst) + " has more than four inputs");
      s[pin] = (uint32_t)src;
      s[0]++;
      indeg[dst]++;
      e_src.push_back((uint32_t)src);
      e_dst.push_back((uint32_t)dst);
    }
  }

  // Adjacency in insertion order (stable counting sort by source).
  const size_t E = e_src.size();
  std::vector<uint32_t> adj_off(N + 1, 0), adj(E);
  for (size_t k = 0; k < E; ++k) adj_off[e_src[k] + 1]++;
  for (uint32_t t = 0; t < N; ++t) adj_off[t + 1] += adj_off[t];
  {
    std::vector<uint32_t> fill(adj_off.begin(), adj_off.end() - 1);
    for (size_t k = 0; k < E; ++k) adj[fill[e_src[k]]++] = e_dst[k];
  }

  // Kahn FIFO seeded with PIs in id order (fsim/simulation.cpp:718-738).
  std::vector<uint32_t> order;
  order.reserve(N);
  for (uint32_t i = 0; i < nPI; ++i) order.push_back(i);
  for (size_t head = 0; head < order.size(); ++head) {
    uint32_t u = order[head];
    for (uint32_t k = adj_off[u]; k < adj_off[u + 1]; ++k) {
      uint32_t v = adj[k];
      if (--indeg[v] == 0) order.push_back(v);
    }
  }
  // POs removed and re-appended in id order (fsim/simulation.cpp:742-751).
  order.erase(std::remove_if(order.begin(), order.end(),
                             [&](uint32_t x) { return x >= nPI && x < nPI + nPO; }),
              order.end());
  for (uint32_t i = 0; i < nPO; ++i) order.push_back(nPI + i);
  if (order.size() != N)
    tk.fail(std::to_string(N - order.size()) +
            " element(s) are not reachable from the PIs (missing fanin or a cycle)");

  // Gate types (fsim/simulation.cpp:760-772).
  std::vector<uint8_t> ftype(N);
  for (uint32_t i = 0; i < nPI; ++i) ftype[i] = G_PI;
  for (uint32_t i = nPI; i < nPI + nPO; ++i) ftype[i] = G_PO;
  for (uint32_t i = nPI + nPO; i < N; ++i) {
    uint64_t t = tk.u64("gate type");
    if (t > 8) tk.fail("gate type " + std::to_string(t) + " outside 0..8");
    ftype[i] = (uint8_t)t;
  }

  nl.tpg.assign(N, 0);
  for (uint32_t i = 0; i < N; ++i) nl.tpg[order[i]] = i;

  // Fanin CSR in topological order: slots 1..count (fsim/simulation.cpp:851-877).
  nl.type.assign(N, 0);
  nl.fi_off.assign(N + 1, 0);
  nl.fi_idx.clear();
  nl.fi_idx.reserve(E);
  for (uint32_t t = 0; t < N; ++t) {
    uint32_t f = order[t];
    nl.type[t] = ftype[f];
    nl.fi_off[t] = (uint32_t)nl.fi_idx.size();
    if (t >= nPI) {
      const uint32_t* s = &slot[(size_t)f * 5];
      for (uint32_t j = 1; j <= s[0]; ++j) nl.fi_idx.push_back((uint32_t)nl.tpg[s[j]]);
      uint32_t cnt = s[0];
      if (cnt == 0) tk.fail("element " + std::to_string(f) + " has no input");
      if (ftype[f] == G_MUX && cnt < 3)
        tk.fail("MUX " + std::to_string(f) + " has fewer than three inputs");
    }
  }
  nl.fi_off[N] = (uint32_t)nl.fi_idx.size();
  finalize_netlist(nl);
}

void parse_flst(const char* text, size_t len, const Netlist& nl, std::vector<Fault>& out) {
  Tok tk{text, text + len, "flst"};
  const bool pins = tk.peek_word("@pins");
  uint64_t F = tk.u64("fault count");
  if (F > (1ull << 32)) tk.fail("fault count out of range");
  out.clear();
  out.reserve(F);
  for (uint64_t i = 0; i < F; ++i) {
    uint64_t id = tk.u64("fault site");
    uint64_t v = tk.u64("fault value");
    uint64_t pin = pins ? tk.u64("fault pin") : 0;
    if (id >= nl.N) tk.fail("fault site " + std::to_string(id) + " out of range");
    uint32_t site = (uint32_t)nl.tpg[id];  // fsim/simulation.cpp:952
    if (pin > nl.fanin_count(site))
      tk.fail("fault pin " + std::to_string(pin) + " exceeds the inputs of element " +
              std::to_string(id));
    out.push_back(Fault{site, (uint8_t)pin, (uint8_t)(v ? 1 : 0)});
  }
}

void parse_ptn(const char* text, size_t len, const Netlist& nl, Patterns& out) {
  Tok tk{text, text + len, "ptn"};
  out = Patterns();
  out.P = tk.u64("pattern count");
  out.W = (out.P + 63) / 64;  // fsim/simulation.cpp:962
  if (out.W * nl.n_pi > (1ull << 36)) tk.fail("pattern block too large");
  out.words.resize(out.W * nl.n_pi);
  for (uint64_t i = 0; i < out.W * nl.n_pi; ++i) out.words[i] = tk.u64("pattern word");
}

}  // namespace fsimb
