// Batch executor shared by the batch API and the serving loop: lays out many
// (circuit, faults, patterns) jobs in device memory and launches the batched
// kernels over all of them.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/fsimb.h"
#include "fsimb_internal.h"
#include "fsimb_kernels.cuh"
#include "fsimb_netlist.h"
#include "fsimb_plan.h"

namespace fsimb {

// Sweep launch shape: words per item, CTA size, target CTAs per SM.
struct ClassShape {
  int M;
  int threads;
  int occ;
};

// One job of a batch.
struct BatchJob {
  const Netlist* nl = nullptr;
  const Plan* plan = nullptr;
  const Schedule* sched = nullptr;  // schedule at M
  const Patterns* pats = nullptr;
  uint64_t F = 0;
  int M = 4;
  int cls = 0;      // sweep class (index into the layout's shapes)
  // resident: the circuit arrays (type, fi_off, fi_idx, level, lvl, blob,
  // li_off, li) are dev's, already on the device.  good_resident:
  // dev.good holds the job's good-machine tiles; no patterns are uploaded and
  // no good machine runs for it.
  bool resident = false;
  bool good_resident = false;
  BatchCirc dev{};
};

// Device bytes of a wave's blocks (what BatchExec::layout asks for).
struct WaveBytes {
  uint64_t stat = 0, work = 0, res = 0, desc = 0, ctl = 0;
};

struct SweepClass {
  int id = 0;  // index into the layout's shapes
  ClassShape shape{0, 0, 0};
  std::vector<uint32_t> circ_ids;   // members, in launch order
  uint32_t queue_base = 0;          // their work counters: d_ctl words 1 + queue_base + j
  unsigned long long n_items = 0;
  double work = 0;        // gate-words its sweeps evaluate (launch order)
  uint32_t max_live = 0;  // slots of the largest schedule in the class
  uint32_t widest = 0;    // largest level block of gate records in the class, 16-byte units
  uint32_t vals_bytes = 0, rec_buf = 0;
  size_t smem = 0;
  int threads = 0, blocks = 0;
};

// Device bytes of a job's work arena: good values (unless resident), sweep
// outputs, sensitivities.
uint64_t batch_job_work_bytes(const BatchJob& j, bool first_tile_only);
// Device bytes of a job's uploaded arrays (circuit and schedule unless
// resident, plan, patterns unless the good values are resident).
uint64_t batch_job_static_bytes(const BatchJob& j);
// The exact sizes layout() asks for, and one job's share of them (the wave's
// sizes are at most the sum of its jobs' shares plus batch_wave_bytes({})).
WaveBytes batch_wave_bytes(const std::vector<BatchJob>& jobs, bool first_tile_only);
WaveBytes batch_job_bytes(const BatchJob& j, bool first_tile_only);

class BatchExec {
 public:
  int n_sms = 0;
  size_t smem_optin = 0, smem_per_sm = 0;

  DevBuf d_static, d_desc, d_work, d_res;
  DevBuf d_ctl;  // [0]: error flag; then one work counter per swept circuit
  PinnedBuf h_static, h_desc, h_res;

  std::vector<BatchCirc> circs;
  std::vector<uint64_t> res_off;
  std::vector<BatchGoodSeg> segs;
  std::vector<uint32_t> level_first_seg;
  std::vector<unsigned long long> level_units;
  std::vector<unsigned long long> ffr_prefix, exact_prefix;
  std::vector<SweepClass> classes;
  unsigned long long ffr_units = 0, exact_units = 0, good_units = 0;
  uint64_t F_total = 0, fault_patterns = 0, dense_gate_words = 0, sweep_alg_bytes = 0,
           good_gate_words = 0;
  uint32_t n_circ = 0;
  bool tile0 = false;
  uint64_t static_bytes = 0, desc_bytes = 0;
  uint64_t ctl_bytes = 256;  // error flag + one work counter per swept circuit
  BatchSweepParams params{};  // launch parameters being built (32 KB)
  size_t smem_attr[4] = {0, 0, 0, 0};  // dynamic smem limit set per words-per-item kernel
  cudaEvent_t* class_events = nullptr;  // direct launches: recorded after each class
  // Classes run as concurrent branches (one stream each), so CTAs of small
  // circuits can share SMs with the CTAs of large ones.
  bool concurrent = true;
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> branch_done;
  cudaEvent_t fork_ev = nullptr;

  const BatchCirc* dd_circs = nullptr;
  const BatchGoodSeg* dd_segs = nullptr;
  const unsigned long long* dd_ffr_prefix = nullptr;
  const unsigned long long* dd_exact_prefix = nullptr;
  unsigned long long* d_count = nullptr;
  unsigned long long* d_first = nullptr;
  uint8_t* d_lastflag = nullptr;

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  uint64_t graph_launches = 0;

  ~BatchExec() { release(); }
  void release();
  uint64_t device_bytes() const;
  // Lays out the jobs: uploads what is not resident, carves the work arena
  // (synchronises `s` before returning).  first_tile_only: only tile 0 of
  // each job (the autotuner's sample).
  void layout(const std::vector<BatchJob>& jobs, const std::vector<ClassShape>& shapes,
              bool first_tile_only, cudaStream_t s);
  // Packs the jobs' static arrays into the pinned staging block and copies it
  // to the device (the layout's pointers stay valid: same jobs, same sizes).
  // Returns the bytes copied.
  uint64_t upload_static(const std::vector<BatchJob>& jobs, cudaStream_t s);
  // New CTA size / CTAs per SM for the laid-out classes.
  void relaunch_shapes(const std::vector<ClassShape>& shapes);
  // Record buffer, shared memory, CTA size and grid of a class for a shape.
  void size_class(SweepClass& k, const ClassShape& sh);
  // Sets each class's dynamic shared-memory limit on its kernel (a
  // per-kernel attribute other launch sequences may have changed).
  void apply_attributes();
  // Enqueues the launch sequence; returns the number of kernels.  With
  // with_events, ev[0] is recorded after the good machine, ev[1] after the sweeps.
  uint64_t enqueue(cudaStream_t s, bool good_only, bool with_events, cudaEvent_t* ev);
  // only >= 0: the class with that id alone.
  uint64_t enqueue_sweeps(cudaStream_t s, int only = -1);
  // All classes as branches forked from and joined into s; class_end[ci]
  // (if given) is recorded when class ci ends.
  uint64_t enqueue_sweeps_concurrent(cudaStream_t s, cudaEvent_t* class_end);
  // Captures the sequence on capture_stream once, then launches the graph on s.
  uint64_t run_graph(cudaStream_t capture_stream, cudaStream_t s);
  void invalidate_graph();
  // Copies the per-fault counters and the error flag to the host (synchronises s).
  void fetch(cudaStream_t s, int* kerr);
  // The same copies, queued on s without waiting; read_err() once they ran.
  void fetch_async(cudaStream_t s);
  int read_err() const;
  void results(size_t i, const BatchJob& j, fsimb_fault_result* out) const;
  uint64_t items() const;
};

}  // namespace fsimb
