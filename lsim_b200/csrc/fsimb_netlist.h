// Host-side netlist, fault-list and pattern model of the stuck-at fault
// simulator.  Everything here follows the semantics of LSIM's CPU simulator
// (fsim/simulation.cpp), which is the behaviour the GPU path must reproduce
// bit for bit:
//
//   * element order  = Kahn FIFO order seeded with the PIs in file-id order,
//                      POs removed and re-appended in file-id order
//                      (fsim/simulation.cpp:718-751);
//   * fanin order    = pin-slot table, slots 1..count (fsim/simulation.cpp:684-711,
//                      851-877), pin 5 (MUX select) remapped to slot 3;
//   * levels         = PIs 0, gates 1+max(fanin), POs max+1
//                      (fsim/simulation.cpp:882-916), raised to stay sorted
//                      in element order where pin-slot gaps break that;
//   * faults         = file id -> topological index, value 0 / ~0
//                      (fsim/simulation.cpp:943-959);
//   * patterns       = ceil(P/64) rows of nPI words (fsim/simulation.cpp:961-976).
//
// Inputs that the reference accepts only with undefined behaviour are rejected
// with a message instead (see validate notes in fsimb_netlist.cpp).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace fsimb {

// Same numbering as GateType in fsim/base_ppg.hpp:19-32 (PI/PO follow CLKBUF).
enum GateType : uint8_t {
  G_INV = 0,
  G_AND = 1,
  G_OR = 2,
  G_XOR = 3,
  G_NAND = 4,
  G_NOR = 5,
  G_XNOR = 6,
  G_MUX = 7,
  G_CLKBUF = 8,
  G_PI = 9,
  G_PO = 10,
};

struct Netlist {
  uint64_t n_pi = 0, n_po = 0, n_gates = 0, n_wires = 0;
  uint32_t N = 0;                 // n_pi + n_gates + n_po
  uint32_t n_levels = 0;          // max PO level + 1 (size of per_level)
  std::vector<uint8_t> type;      // [N] by topological index
  std::vector<uint32_t> level;    // [N]
  std::vector<uint32_t> fi_off;   // [N+1] fanin CSR, pin order
  std::vector<uint32_t> fi_idx;   // [E]
  std::vector<uint32_t> fo_off;   // [N+1] fanout CSR (one entry per consumer pin)
  std::vector<uint32_t> fo_idx;   // [E] consumer topological index, ascending
  std::vector<uint8_t> fo_pin;    // [E] position of the edge in the consumer's fanin list
  std::vector<uint64_t> tpg;      // [N] file id -> topological index
  std::vector<uint64_t> per_level;  // [n_levels] element count per level
  std::vector<uint32_t> level_off;  // [n_levels+1] first topological index of each level
  // The reference's levels and per-level counts where they differ from
  // `level` / `per_level` (element order not level-sorted by them); empty
  // otherwise.  `level` is then the schedule level: 1 + max fanin level and
  // at least the level of the element before, so level ranges stay
  // contiguous in element order.
  std::vector<uint32_t> ref_level;
  std::vector<uint64_t> ref_per_level;

  uint32_t fanin_count(uint32_t e) const { return fi_off[e + 1] - fi_off[e]; }
};

// One stuck-at fault.  pin == 0: output (stem) of element `site`; pin k >= 1:
// the k-th input (1-based position in the fanin list) of element `site`.
// The reference .flst format can only express pin == 0.
struct Fault {
  uint32_t site;
  uint8_t pin;
  uint8_t value;  // 0 = SA0, 1 = SA1
};

struct Patterns {
  uint64_t P = 0;                // number of patterns
  uint64_t W = 0;                // rounds = ceil(P/64)
  std::vector<uint64_t> words;   // [W][n_pi] row-major, round-major
  // Valid low bits in round rd (fsim/simulation.cpp:115-118).
  uint32_t bits(uint64_t rd) const {
    return (P / (64 * (rd + 1))) ? 64u : (uint32_t)(P % 64);
  }
};

// Parse errors throw ParseError; the C ABI turns them into status codes.
struct ParseError {
  std::string msg;
};

// .ckt reader + levelizer.
void parse_ckt(const char* text, size_t len, Netlist& out);
// .flst reader.  Standard form: "F" then F pairs "file_id value".  Extended
// form (pin faults): leading token "@pins", then "F" and F triples
// "file_id value pin".
void parse_flst(const char* text, size_t len, const Netlist& nl, std::vector<Fault>& out);
// .ptn reader: "P" then ceil(P/64) rows of n_pi decimal words.  Rows are kept
// in file order (round r = row r); the reference stores row r at round
// tpg[r], which is the identity whenever ceil(P/64) <= n_pi.
void parse_ptn(const char* text, size_t len, const Netlist& nl, Patterns& out);

// Builds the derived arrays (levels, fanout CSR, level offsets) after the
// fanin CSR and types are set.  Used by the reader and by generators that
// build a Netlist directly.
void finalize_netlist(Netlist& nl);

}  // namespace fsimb
