// Seeded synthetic workloads: levelized combinational DAGs written in the
// .ckt format, stuck-at fault lists (.flst, plain or with pin faults) and
// bit-packed pattern blocks (.ptn).  The text conventions follow the
// reference's generators (fsim/circuit_generator.py:101-113,
// fsim/generate_fault_patterns.py:26-94): element ids PIs, then POs, then
// gates; pins 1..3 (5 for a MUX select); pattern chunks MSB-first.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "fsimb_netlist.h"

namespace fsimb {

struct GenConfig {
  uint64_t seed = 0;
  uint32_t n_gates = 2000, n_pi = 64, n_po = 64, n_levels = 30;
  uint32_t window = 4;          // inputs come from at most this many levels back
  double p_fanin3 = 0.5;        // multi-input gates: P(3 inputs), else 2
  uint32_t type_mask = 0x17F;   // allowed GateType values (bit t); default all but MUX
  double hub_frac = 0.0;        // fraction of gates with a large fanout target
  uint32_t hub_fo_min = 8, hub_fo_max = 64;
  uint32_t fo_min = 1, fo_max = 3;  // fanout target of non-hub gates (hub mode only)
  double p_unused = 0.5;        // extra inputs: P(take a still-unused source)
  int shuffle_ids = 1;          // randomise the gate file ids
};

// Writes the circuit as .ckt text.
std::string generate_ckt(const GenConfig& cfg);

struct PatternConfig {
  uint64_t seed = 0;
  uint64_t n_patterns = 4096;
  double biased_pi_frac = 0.0;  // fraction of PIs drawn with P(1) = p_one_biased
  double p_one_biased = 0.2;
};

// Pattern words [W][n_pi]; high bits of a partial last round are zero.
void generate_patterns(const PatternConfig& cfg, uint64_t n_pi, Patterns& out);
std::string write_ptn(const Patterns& p, uint64_t n_pi);

// Fault lists over a parsed netlist.
enum FaultListKind { FL_OUTPUTS = 0, FL_OUTPUTS_AND_PINS = 1, FL_COLLAPSED = 2 };
void build_fault_list(const Netlist& nl, FaultListKind kind, std::vector<Fault>& out);
// Serialises faults with file ids; uses the extended "@pins" form when any
// fault is on an input pin (or when force_pins is set).
std::string write_flst(const Netlist& nl, const std::vector<Fault>& faults, bool force_pins);

}  // namespace fsimb
