// Host-side compilation of a netlist + fault list into the device data layout
// used by the B200 kernels.
//
// Layout in HBM (all arrays indexed by the reference's topological index):
//   type[N]            u8 gate type
//   fi_off[N+1], fi_idx[E]   fanin CSR in pin order (good-machine kernel)
//   sweep blocks       per level one block of gate records (the level's
//                      order of evaluation), 16-byte aligned:
//                        plain records, 8 bytes: 15-bit shared-memory slots
//                        of up to three fanins and of the output, and a
//                        4-bit gate class (PlainClass) -- every non-MUX gate
//                        with 1-3 inputs that feeds other gates and no PO;
//                        wide records, 16 bytes (SweepRec): everything else
//                        that must be evaluated (PO drivers, MUX, 4 inputs).
//                      Gates that feed nothing are left out.  Within each
//                      part the order is by class, and every group of G
//                      consecutive positions has pairwise different slot
//                      residues mod G for each fanin and for the output
//                      wherever the host found such groups, so the group's
//                      shared-memory accesses hit distinct banks
//   lvl[L]             (block offset in 16-byte units, plain count, wide
//                      count, block size in 16-byte units)
//   li_off[L+1], li[]  (element, slot) pairs live when a sweep starts at
//                      level L (read from the good values at start)
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
constexpr uint32_t kNoSlot = 0xFFFFFFFFu;
constexpr uint32_t kMaxSlots = 32767;   // slots are 15-bit in the plain gate records

// Plain gate records: classes of the gate function (a compile-time body in
// the sweep kernel each).  One-input gates are BUF (AND, OR, XOR, CLKBUF) or
// INV (INV, NAND, NOR, XNOR).  kPNop pads a level's plain part to a group
// boundary and does nothing.
enum PlainClass : uint32_t {
  kPBuf = 0, kPInv, kPAnd2, kPNand2, kPOr2, kPNor2, kPXor2, kPXnor2,
  kPAnd3, kPNand3, kPOr3, kPNor3, kPXor3, kPXnor3, kPlainClasses, kPNop = 15
};
// Classes that share one sweep body, which reads the class's input and
// output inversions from the class code at run time: one input, AND family
// (AND, NAND, OR, NOR) with two and with three inputs, XOR family with two
// and with three inputs.  The host groups records by body, not by class:
// larger groups leave fewer repeated bank residues and fewer class
// boundaries inside a warp.
inline uint32_t plain_body(uint32_t cls) {
  return cls < kPAnd2 ? 0u : cls < kPXor2 ? 1u : cls < kPAnd3 ? 2u : cls < kPXor3 ? 3u : 4u;
}
// Bits [0,15) fanin 0, [15,30) fanin 1, [30,45) fanin 2, [45,60) output
// slot, [60,64) class.
inline uint64_t plain_rec(uint32_t f0, uint32_t f1, uint32_t f2, uint32_t out, uint32_t cls) {
  return (uint64_t)f0 | ((uint64_t)f1 << 15) | ((uint64_t)f2 << 30) | ((uint64_t)out << 45) |
         ((uint64_t)cls << 60);
}

// One level of the sweep order (see "sweep blocks" above).
struct LevelDesc {
  uint32_t off16;    // block offset in 16-byte units
  uint32_t n_plain;  // plain records (8 bytes each, first)
  uint32_t n_wide;   // wide records (16 bytes each, after the plain part padded to 16 bytes)
  uint32_t n16;      // block size in 16-byte units
};

// SweepRec::meta bit fields
constexpr uint32_t kRecTypeMask = 15u;     // bits 0-3: gate type
constexpr int kRecNfShift = 4;             // bits 4-5: fan-in - 1
constexpr uint32_t kRecPo = 1u << 6;       // drives a PO
constexpr uint32_t kRecHasSlot = 1u << 7;  // has gate consumers (value stored)
constexpr int kRecClassShift = 8;          // bits 8-11: gate class (sweep code path)
constexpr uint32_t kRecIi = 1u << 12;      // invert inputs (OR, NOR)
constexpr uint32_t kRecIo = 1u << 13;      // invert output (INV, OR, NAND, XNOR)
// Gate classes: 0-3 AND family with 1-4 inputs, 4-6 XOR family with 2-4
// inputs, 7 MUX with 3 inputs, 8 any other combination (generic path).
constexpr uint32_t kClassGeneric = 8;

// InjRec::mode bit fields
constexpr uint32_t kInjStuck = 1u;      // 0: flip the element's word, 1: stuck value
constexpr uint32_t kInjReachesPo = 2u;  // the element is, or drives, a PO

// Observability source of an FFR root.
constexpr uint32_t kObsZero = 0xFFFFFFFEu;  // root reaches no PO
constexpr uint32_t kObsOne = 0xFFFFFFFFu;   // root is / drives a PO

struct SweepRec {  // wide gate record
  uint16_t fs[4];  // fanin slots
  uint16_t slot;   // own slot (valid with kRecHasSlot)
  uint16_t meta;
  uint32_t elem;   // topological index
};
static_assert(sizeof(SweepRec) == 16, "SweepRec is one 16-byte load");

struct RootRec {
  uint32_t root;
  uint32_t obs;        // sweep index, kObsZero or kObsOne
  uint32_t mem_begin;  // into members
  uint32_t mem_end;
  uint32_t flt_begin;  // into traced faults
  uint32_t flt_end;
  uint32_t slot;       // compact sensitivity slot of the root: members.size() + root index
  uint32_t pad;
};

struct MemberRec {  // internal FFR element e, its consumer p and pin position
  uint32_t e;
  uint32_t p;
  uint32_t pin;
  uint32_t p_slot;  // compact sensitivity slot of p (a member's slot is its index in members)
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
  uint32_t mode;    // kInjStuck | kInjReachesPo
  uint32_t value;
};

struct Plan {
  uint32_t N = 0, n_pi = 0, n_gates = 0, n_po = 0;
  uint32_t n_levels = 0;
  uint32_t max_gate_level = 0;       // highest level holding a non-PO element
  uint32_t max_live = 0;             // slots needed without residue constraints
  uint32_t max_level_width = 0;
  uint64_t dense_sweep_gates = 0;    // sum over sweeps of gates evaluated
  uint64_t dense_sweep_bytes = 0;    // sum over sweeps of 8*(fanin+1) per evaluated gate, per word
  // [N+1] prefix sums of 8*(effective fanin+1) over the elements a sweep
  // evaluates (gates that feed a gate or a PO)
  std::vector<uint64_t> nfp_prefix;
  std::vector<uint32_t> eval_prefix; // [N+1] prefix counts of those elements
  std::vector<uint32_t> level_off;   // [n_levels+1]
  std::vector<uint32_t> maxfo_level; // [N] highest non-PO consumer level (0 if none)
  std::vector<uint8_t> gate_fo;      // [N] has a non-PO consumer
  std::vector<uint8_t> po_drv;       // [N] drives a PO
  // traced faults
  std::vector<RootRec> roots;
  std::vector<MemberRec> members;
  std::vector<TracedRec> traced;
  std::vector<uint32_t> traced_slot;  // compact sensitivity slot of each traced fault's element
  // sweeps: first n_stem_sweeps are root flips, the rest exact faults
  std::vector<InjRec> sweeps;
  uint32_t n_stem_sweeps = 0;
  std::vector<uint32_t> exact_fault;  // fault index of each exact sweep
  std::vector<uint32_t> sweep_root;   // root record of each stem sweep
  bool has_mux = false;
};

// The fault-independent part of a plan, built once per circuit: `base` holds
// the circuit fields of Plan (sizes, levels, fanout facts, live-value peak,
// byte prefix sums; no roots or sweeps), plus what classifying a fault list
// needs: MUX-below flags, the FFR root of every element and the members of
// every FFR (element-descending, consumer first).
struct CircuitPlan {
  Plan base;
  std::vector<uint8_t> mux_below;   // [N] some consumer path reaches a MUX
  std::vector<uint32_t> root;       // [N] FFR root
  std::vector<uint32_t> ffr_off;    // [N+1] members of the FFR rooted at r
  std::vector<MemberRec> ffr_mem;
  std::vector<uint32_t> ffr_local;  // [N] position of a member within its FFR's list
};

// Per-level evaluation order and shared-memory slots for one residue group
// size G (16 / words per item).
struct Schedule {
  uint32_t G = 0;
  uint32_t max_live = 0;             // slots (multiple of G)
  std::vector<uint64_t> blob;        // level blocks (8-byte units; each block 16-byte aligned)
  std::vector<LevelDesc> lvl;        // [n_levels+1]; levels 1..max_gate_level used
  uint32_t max_block16 = 0;          // largest level block, 16-byte units
  std::vector<uint32_t> li_off;      // [n_levels+1]
  std::vector<uint32_t> li;          // pairs (element, slot)
  uint64_t conflict_groups = 0;      // group accesses whose slots repeat a residue
  uint64_t access_groups = 0;        // group accesses (fanin loads + stores)
  uint64_t bytes() const {
    return blob.size() * 8 + lvl.size() * sizeof(LevelDesc) + li_off.size() * 4 + li.size() * 4;
  }
};

// 0: AND family (AND, NAND, OR, NOR, INV, CLKBUF, PO), 1: XOR family, 2: MUX.
uint32_t gate_family(uint8_t type);
uint32_t gate_class(uint8_t type, uint32_t fanin);
void build_plan(const Netlist& nl, const std::vector<Fault>& faults, Plan& plan);
void build_circuit_plan(const Netlist& nl, CircuitPlan& cplan);
// Roots, members, traced faults and sweeps of a fault list; the circuit's
// per-element vectors (maxfo_level, gate_fo, po_drv, nfp_prefix) stay in
// cplan.base and are left empty in `plan`.  Costs O(faults log faults +
// members of the FFRs the faults touch).
void build_fault_plan(const Netlist& nl, const CircuitPlan& cplan, const std::vector<Fault>& faults,
                      Plan& plan);
// Class of a plain record, or kPlainClasses when the gate needs a wide one.
uint32_t plain_class(uint8_t type, uint32_t eff_fanin);
// G in {2, 4, 8, 16}.  A schedule that needs more than kMaxSlots slots
// reports max_live > kMaxSlots and leaves blob and li empty.
void build_schedule(const Netlist& nl, const Plan& plan, uint32_t G, Schedule& out);

}  // namespace fsimb
