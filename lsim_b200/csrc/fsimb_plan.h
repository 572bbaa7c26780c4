// Host-side compilation of a netlist + fault list into the device data layout
// used by the B200 kernels.
//
// Layout in HBM (all arrays indexed by the reference's topological index):
//   type[N]            u8 gate type
//   fi_off[N+1], fi_idx[E]   fanin CSR in pin order (good-machine kernel)
//   sw_fslot[N]        uint4: shared-memory slot of each of up to 4 fanins
//   sw_meta[N]         u32: own slot | has_slot | drives_po | nfanin-1 | type
//   li_off[L+1], li_elem[]   elements whose value is live when a sweep starts
//                            at level L (read from the good values at start)
//   good[tile][N][32]  u64 good-machine words, 32 words (2048 patterns) per tile
//
// Fault handling:
//   * fanout-free regions (FFRs): every element with exactly one consumer
//     belongs to the FFR of that consumer; all others are FFR roots;
//   * faults whose downstream logic is bitwise (no MUX) are "traced": their
//     detection word is  sens(line -> root) & (good(line) ^ stuck) & obs(root)
//     where sens is computed by backward critical-path tracing inside the
//     FFR and obs(root) by one sweep per root that flips the root's value;
//   * faults with a MUX downstream are "exact": one sweep per fault with the
//     stuck value injected, since the reference's MUX uses a word-level
//     logical not (fsim/simulation.cpp:1056) that is not bitwise.
#pragma once

#include <cstdint>
#include <vector>

#include "fsimb_netlist.h"

namespace fsimb {

constexpr uint32_t kTileWords = 32;  // words per tile = lanes of a warp
constexpr uint32_t kNoSlot = 0x7FFFFFu;

// sw_meta bit fields
constexpr uint32_t kMetaSlotMask = 0x7FFFFFu;
constexpr uint32_t kMetaHasSlot = 1u << 23;
constexpr uint32_t kMetaPo = 1u << 24;
constexpr int kMetaNfShift = 25;   // 2 bits: nfanin - 1
constexpr int kMetaTypeShift = 27; // 4 bits

// Observability source of an FFR root.
constexpr uint32_t kObsZero = 0xFFFFFFFEu;  // root reaches no PO
constexpr uint32_t kObsOne = 0xFFFFFFFFu;   // root is / drives a PO

struct RootRec {
  uint32_t root;
  uint32_t obs;        // sweep index, kObsZero or kObsOne
  uint32_t mem_begin;  // into members
  uint32_t mem_end;
  uint32_t flt_begin;  // into traced faults
  uint32_t flt_end;
  uint32_t pad[2];
};

struct MemberRec {  // internal FFR element e, its consumer p and pin position
  uint32_t e;
  uint32_t p;
  uint32_t pin;
  uint32_t pad;
};

struct TracedRec {  // one traced fault
  uint32_t fault;   // index into the caller's fault list
  uint32_t elem;    // output fault: the element; pin fault: the gate
  uint32_t pin;     // 0 = output, k = k-th input
  uint32_t value;   // 0 / 1
};

struct InjRec {     // sweep injection: flip (stem) or stuck (exact fault)
  uint32_t elem;
  uint32_t pin;     // exact faults: 0 output, k input; flips: 0
  uint32_t mode;    // 0 flip, 1 stuck
  uint32_t value;
};

struct Plan {
  uint32_t N = 0, n_pi = 0, n_gates = 0, n_po = 0;
  uint32_t n_levels = 0;
  uint32_t max_gate_level = 0;       // highest level holding a non-PO element
  uint32_t max_live = 0;             // shared-memory slots needed by a sweep
  uint32_t max_level_width = 0;
  uint64_t dense_sweep_gates = 0;    // sum over sweeps of gates evaluated
  uint64_t dense_sweep_bytes = 0;    // sum over sweeps of 8*(fanin+1) per evaluated gate, per word
  std::vector<uint64_t> nfp_prefix;  // [N+1] prefix sums of 8*(effective fanin+1)
  std::vector<uint32_t> level_off;   // [n_levels+1]
  std::vector<uint32_t> fslot;       // [4N]
  std::vector<uint32_t> meta;        // [N]
  std::vector<uint32_t> li_off;      // [n_levels+1]
  std::vector<uint32_t> li_elem;
  std::vector<uint32_t> maxfo_level; // [N] highest non-PO consumer level (0 if none)
  // traced faults
  std::vector<RootRec> roots;
  std::vector<MemberRec> members;
  std::vector<TracedRec> traced;
  // sweeps: first n_stem_sweeps are root flips, the rest exact faults
  std::vector<InjRec> sweeps;
  uint32_t n_stem_sweeps = 0;
  std::vector<uint32_t> exact_fault;  // fault index of each exact sweep
  std::vector<uint32_t> sweep_root;   // root record of each stem sweep
  bool has_mux = false;
};

void build_plan(const Netlist& nl, const std::vector<Fault>& faults, Plan& plan);

}  // namespace fsimb
