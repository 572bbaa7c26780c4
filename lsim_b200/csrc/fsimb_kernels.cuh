// Device kernels of the B200 stuck-at fault simulator.  All arithmetic is
// bitwise on 64-bit words (64 patterns per word); no tensor cores are
// involved because gate evaluation is not a contraction.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fsimb_plan.h"

namespace fsimb {

struct GoodArgs {
  const uint8_t* type;
  const uint32_t* fi_off;
  const uint32_t* fi_idx;
  const uint64_t* pwords;  // [W][n_pi]
  uint64_t* good;          // [tiles][N][32]
  uint32_t n_pi, N;
  uint32_t lo, hi;         // element range of one level
  uint32_t W, W_pad;       // real and padded word counts
};

struct SweepArgs {
  const uint4* blob;       // level blocks of gate records (see fsimb_plan.h)
  const uint4* lvl;        // LevelDesc per level
  const uint32_t* level;   // element -> level
  const uint32_t* li_off;
  const uint32_t* li;      // (element, slot) pairs
  const uint32_t* fi_off;
  const uint32_t* fi_idx;
  const uint8_t* type;
  const InjRec* inj;
  const uint32_t* list;    // sweep indices to run (nullptr: 0..n_list-1)
  uint32_t n_list;
  uint32_t max_gate_level;
  uint32_t N;
  const uint64_t* good;    // this tile: [N][32]
  uint64_t* out;           // this tile: [n_sweeps][32] OR of PO differences
  int* queue;              // work counter for this launch
  uint32_t vals_bytes;     // shared memory for values (multiple of 16)
  uint32_t rec_buf;        // 16-byte units per staging buffer (2 buffers follow the values)
  int* err;                // set to 1 if a bounded wait gave up
  uint64_t wait_ns;        // time limit of one wait for a record copy
  uint32_t wait_test;      // 1: the first CTA waits on a barrier no copy completes (test hook)
};

// Sweep of circuits whose live values do not fit in shared memory.
struct SweepWideArgs {
  const uint32_t* level;     // element -> level
  const uint32_t* level_off; // element offsets per level
  const uint32_t* fi_off;
  const uint32_t* fi_idx;
  const uint8_t* type;
  const uint8_t* eflag;      // bit 0: evaluated in sweeps, bit 1: drives a PO
  const InjRec* inj;
  const uint32_t* list;      // sweep indices to run (nullptr: 0..n_list-1)
  uint32_t n_list;
  uint32_t max_gate_level;
  uint32_t N;
  const uint64_t* good;      // this tile: [N][32]
  uint64_t* out;             // this tile: [n_sweeps][32]
  int* queue;
  uint64_t* gvals;           // [blocks][N][M] values of each CTA's item
};

struct FfrArgs {
  const RootRec* roots;
  const uint32_t* list;    // root indices to process (nullptr: all)
  uint32_t n_list;
  const MemberRec* members;
  const TracedRec* traced;
  const uint32_t* fi_off;
  const uint32_t* fi_idx;
  const uint8_t* type;
  const uint64_t* good;    // tile [N][32]
  const uint64_t* obs;     // tile [n_sweeps][32]
  uint64_t* sens;          // scratch [N][32]
  uint32_t tile, W;
  uint64_t P;
  int drop;                // skip faults whose count reached n_detect in an earlier tile
  uint32_t n_detect;       // >= 1
  unsigned long long* count;
  unsigned long long* first;
  uint8_t* lastflag;
};

struct ExactArgs {
  const uint32_t* exact_fault;
  const uint32_t* list;    // exact indices to process (nullptr: all)
  uint32_t n_exact;
  uint32_t first_sweep;    // index of the first exact sweep
  const uint64_t* out;     // tile [n_sweeps][32]
  uint32_t tile, W;
  uint64_t P;
  int drop;
  uint32_t n_detect;
  unsigned long long* count;
  unsigned long long* first;
  uint8_t* lastflag;
};

// Threads [0, n_in_pad) handle roots, the rest exact faults.
struct DropArgs {
  const RootRec* roots;
  const uint32_t* in_list;   // current live roots (nullptr: all)
  uint32_t n_in, n_in_pad;
  const TracedRec* traced;
  const uint32_t* exact_fault;
  const uint32_t* exact_in;  // current live exact indices (nullptr: all)
  uint32_t n_exact_in;
  uint32_t first_exact_sweep;
  const unsigned long long* count;
  uint32_t n_detect;         // a fault survives while its count is below this
  uint32_t* out_roots;       // surviving root indices
  uint32_t* out_sweeps;      // sweeps still needed (stem flips and exact faults)
  uint32_t* out_exact;       // surviving exact indices
  uint32_t* n_out;           // [3]: roots, sweeps, exact
};

// ---------------------------------------------------------------- batches
// One circuit of a batch: device pointers into the batch's concatenated
// arrays and the circuit's sizes.
struct BatchCirc {
  const uint4* blob;
  const uint4* lvl;
  const uint32_t* level;
  const uint32_t* li_off;
  const uint32_t* li;
  const uint32_t* fi_off;
  const uint32_t* fi_idx;
  const uint8_t* type;
  const InjRec* inj;
  const RootRec* roots;
  const MemberRec* members;
  const TracedRec* traced;
  const uint32_t* traced_slot;
  const uint32_t* exact_fault;
  const uint64_t* pwords;        // [W][n_pi]
  uint64_t* good;                // [tiles][N][32]
  uint64_t* out;                 // [tiles][n_sweeps][32]
  uint64_t* sens;                // [tiles][n_slots][32]: members, then roots
  unsigned long long* count;     // per fault
  unsigned long long* first;
  uint8_t* lastflag;
  uint64_t P;
  uint32_t N, n_pi, W, tiles;
  uint32_t n_sweeps, n_stem_sweeps, n_roots, n_exact;
  uint32_t max_gate_level, n_levels;
  uint32_t n_slots, pad;         // sensitivity slots per tile
};

// What the batched sweep reads of one circuit.  A launch carries these in
// its parameters, so the compiler sees them as warp-uniform values.
struct SweepCirc {
  const uint4* blob;
  const uint4* lvl;
  const uint32_t* level;
  const uint32_t* li_off;
  const uint32_t* li;
  const uint32_t* fi_off;
  const uint32_t* fi_idx;
  const uint8_t* type;
  const InjRec* inj;
  const uint64_t* good;  // [tiles][N][32]
  uint64_t* out;         // [tiles][n_sweeps][32]
  uint32_t N, n_sweeps, max_gate_level;
  uint32_t n_items;      // tiles * n_sweeps * (32 / M): (tile, sweep, subtile), tile-major
};

constexpr int kSweepCircsPerLaunch = 300;

struct BatchSweepParams {
  SweepCirc c[kSweepCircsPerLaunch];
  unsigned long long* queue;  // [n_circ] work counters, zero before the launch
  int* err;
  uint64_t wait_ns;
  uint32_t n_circ, vals_bytes, rec_buf;
};
static_assert(sizeof(BatchSweepParams) <= 32000, "kernel parameters are limited to 32,764 bytes");

// A level of the batched good machine: segments (circuit, element range)
// with one warp per (element, tile).
struct BatchGoodSeg {
  uint32_t circ, lo, hi, pad;
  unsigned long long unit0;  // first unit of the segment
};

// Units of the batched tracing kernels: one warp per (circuit, tile, root)
// or (circuit, tile, exact fault); prefix over circuits.
struct BatchUnits {
  const BatchCirc* circs;
  const unsigned long long* unit_prefix;  // [n_circ + 1]
  uint32_t n_circ;
};

void launch_good_batch(const BatchCirc* circs, const BatchGoodSeg* segs, uint32_t n_segs,
                       unsigned long long n_units, cudaStream_t s);
cudaError_t launch_sweep_batch(int M, int threads, int blocks, size_t smem, const BatchSweepParams& p,
                               cudaStream_t s);
cudaError_t sweep_batch_set_smem(int M, size_t smem);
cudaError_t sweep_batch_occupancy(int M, int threads, size_t smem, int* blocks_per_sm);
void launch_ffr_batch(const BatchUnits& u, unsigned long long n_units, cudaStream_t s);
void launch_exact_batch(const BatchUnits& u, unsigned long long n_units, cudaStream_t s);
void launch_init_results_batch(unsigned long long* count, unsigned long long* first, uint8_t* lastflag,
                               uint64_t F, cudaStream_t s);

void launch_good_level(const GoodArgs& a, cudaStream_t s);
// Returns cudaErrorInvalidValue when M is unsupported.
cudaError_t launch_sweep(int M, int threads, int blocks, size_t smem, const SweepArgs& a,
                         cudaStream_t s);
cudaError_t sweep_set_smem(int M, size_t smem);
cudaError_t sweep_occupancy(int M, int threads, size_t smem, int* blocks_per_sm);
// M in {1, 2}; 256 threads per CTA.
cudaError_t launch_sweep_wide(int M, int blocks, const SweepWideArgs& a, cudaStream_t s);
cudaError_t sweep_wide_occupancy(int M, int* blocks_per_sm);
// Time limit of one wait for a record copy, and the shorter one of the wait test.
constexpr uint64_t kWaitLimitNs = 2000000000ull;
constexpr uint64_t kWaitTestNs = 20000000ull;
void launch_ffr(const FfrArgs& a, cudaStream_t s);
void launch_exact(const ExactArgs& a, cudaStream_t s);
void launch_init_results(unsigned long long* count, unsigned long long* first, uint8_t* lastflag,
                         uint32_t F, cudaStream_t s);
void launch_drop(const DropArgs& a, cudaStream_t s);

}  // namespace fsimb
