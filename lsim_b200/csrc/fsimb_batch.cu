// Batched fault simulation: many circuits, each with its own fault list and
// pattern block, simulated together (fsimb_batch_* of include/fsimb.h).
//
// One run is a fixed launch sequence over all member circuits at once:
//   * results init: one launch over the faults of every circuit;
//   * good machine: one k_good_batch launch per level index, holding the
//     elements of that level of every circuit, all tiles of each;
//   * sweeps: one persistent k_sweep_batch launch per words-per-item class,
//     its CTAs pulling (circuit, tile, sweep, subtile) items from one device
//     counter, so circuits of very different sizes share the SMs;
//   * FFR tracing and the exact-fault epilogue: one launch each over all
//     (circuit, tile, root) and (circuit, tile, exact fault) units.
// The sequence is captured into a CUDA graph once and replayed while the
// membership and the shape stay the same.  The sweep shape (words per item,
// CTA size, CTAs per SM) comes from timing candidates on a sample of the
// batch (the autotuner: the first tile of a spread of its circuits) or from
// the plain path's heuristic.
//
// Results equal the plain path's (fsimb_run) for every circuit: the same
// kernels' arithmetic on the same per-circuit data; only the order in which
// tiles accumulate into a fault's counters differs, and those are integer
// sums and minima.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fsimb.h"
#include "fsimb_batch.h"
#include "fsimb_internal.h"
#include "fsimb_kernels.cuh"

using namespace fsimb;

namespace fsimb {

namespace {

int m_slot(int M) { return M == 1 ? 0 : M == 2 ? 1 : M == 4 ? 2 : 3; }

uint64_t align256(uint64_t x) { return (x + 255) & ~255ull; }

// Runs f(i) for i in [0, n) on up to hardware_concurrency threads; the
// first exception a worker raised is rethrown on the calling thread.
template <class F>
void parallel_for(size_t n, F f) {
  const size_t nt = std::min<size_t>(n, std::max(1u, std::thread::hardware_concurrency()));
  if (nt <= 1) {
    for (size_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> ts;
  std::atomic<size_t> next{0};
  std::vector<std::exception_ptr> errs(nt);
  for (size_t t = 0; t < nt; ++t)
    ts.emplace_back([&, t] {
      try {
        for (size_t i = next++; i < n; i = next++) f(i);
      } catch (...) {
        errs[t] = std::current_exception();
        next = n;  // the others stop at their next item
      }
    });
  for (auto& t : ts) t.join();
  for (auto& e : errs)
    if (e) std::rethrow_exception(e);
}

}  // namespace

// ------------------------------------------------------------ BatchExec

uint64_t batch_job_work_bytes(const BatchJob& j, bool first_tile_only) {
  const uint64_t tiles = first_tile_only ? 1 : std::max<uint64_t>(1, (j.pats->W + kTileWords - 1) / kTileWords);
  const uint64_t N = j.plan->N;
  const uint64_t ns = j.plan->sweeps.size();
  const uint64_t slots = j.plan->members.size() + j.plan->roots.size();
  uint64_t b = 0;
  if (!j.good_resident) b += align256(tiles * N * kTileWords * 8);        // good
  b += align256(tiles * std::max<uint64_t>(ns, 1) * kTileWords * 8);      // out
  if (!first_tile_only) b += align256(tiles * std::max<uint64_t>(slots, 1) * kTileWords * 8);  // sens
  return b;
}

uint64_t batch_job_static_bytes(const BatchJob& j) {
  const Netlist& nl = *j.nl;
  const Plan& p = *j.plan;
  uint64_t b = 0;
  auto t = [&](uint64_t bytes) { b += align256(bytes); };
  if (!j.resident) {
    const Schedule& sc = *j.sched;
    t(nl.type.size());
    t(nl.fi_off.size() * 4);
    t(nl.fi_idx.size() * 4);
    t(nl.level.size() * 4);
    t(sc.lvl.size() * sizeof(LevelDesc));
    t(sc.blob.size() * 8);
    t(sc.li_off.size() * 4);
    t(sc.li.size() * 4);
  }
  t(p.sweeps.size() * sizeof(InjRec));
  t(p.roots.size() * sizeof(RootRec));
  t(p.members.size() * sizeof(MemberRec));
  t(p.traced.size() * sizeof(TracedRec));
  t(p.traced_slot.size() * 4);
  t(p.exact_fault.size() * 4);
  if (!j.good_resident) t(j.pats->words.size() * 8);
  return b;
}

uint32_t batch_job_good_segments(const BatchJob& j) {
  if (j.good_resident) return 0;
  uint32_t n = 0;
  for (uint32_t l = 0; l < j.nl->n_levels; ++l) n += j.nl->level_off[l + 1] > j.nl->level_off[l];
  return n;
}

WaveBytes batch_wave_bytes(const std::vector<BatchJob>& jobs, bool first_tile_only) {
  WaveBytes w;
  uint64_t F = 0, segs = 0, swept = 0;
  for (const BatchJob& j : jobs) {
    w.stat += batch_job_static_bytes(j);
    w.work += batch_job_work_bytes(j, first_tile_only);
    F += j.F;
    segs += batch_job_good_segments(j);
    swept += j.plan->sweeps.empty() ? 0 : 1;
  }
  const uint64_t n = jobs.size();
  w.res = std::max<uint64_t>(F, 1) * 17 + 512;
  w.desc = align256(n * sizeof(BatchCirc)) + align256(segs * sizeof(BatchGoodSeg)) + 2 * align256((n + 1) * 8);
  w.ctl = align256((swept + 1) * 8);
  return w;
}

WaveBytes batch_job_bytes(const BatchJob& j, bool first_tile_only) {
  WaveBytes w;
  w.stat = batch_job_static_bytes(j);
  w.work = batch_job_work_bytes(j, first_tile_only);
  w.res = 17 * j.F;
  w.desc = sizeof(BatchCirc) + batch_job_good_segments(j) * sizeof(BatchGoodSeg) + 16;
  w.ctl = 8;
  return w;
}

void BatchExec::release() {
  if (gexec) cudaGraphExecDestroy(gexec);
  if (graph) cudaGraphDestroy(graph);
  gexec = nullptr;
  graph = nullptr;
  for (cudaStream_t x : branch) cudaStreamDestroy(x);
  for (cudaEvent_t e : branch_done) cudaEventDestroy(e);
  if (fork_ev) cudaEventDestroy(fork_ev);
  branch.clear();
  branch_done.clear();
  fork_ev = nullptr;
  for (DevBuf* b : {&d_static, &d_desc, &d_work, &d_res, &d_ctl}) b->release();
  for (PinnedBuf* b : {&h_static, &h_desc, &h_res}) b->release();
}

uint64_t BatchExec::device_bytes() const {
  return d_static.n + d_desc.n + d_work.n + d_res.n + d_ctl.n;
}

uint64_t BatchExec::upload_static(const std::vector<BatchJob>& jobs, cudaStream_t s) {
  uint8_t* hb = h_static.as<uint8_t>();
  char* db = d_static.as<char>();
  uint64_t at = 0;
  auto put = [&](const void* src, uint64_t bytes) -> const void* {
    const uint64_t o = at;
    if (bytes) std::memcpy(hb + o, src, bytes);
    at = o + align256(bytes);
    return db + o;
  };
  for (size_t i = 0; i < jobs.size(); ++i) {
    const BatchJob& j = jobs[i];
    const Netlist& nl = *j.nl;
    const Plan& p = *j.plan;
    BatchCirc& c = circs[i];
    if (j.resident) {  // circuit arrays already on the device
      c.type = j.dev.type;
      c.fi_off = j.dev.fi_off;
      c.fi_idx = j.dev.fi_idx;
      c.level = j.dev.level;
      c.lvl = j.dev.lvl;
      c.blob = j.dev.blob;
      c.li_off = j.dev.li_off;
      c.li = j.dev.li;
    } else {
      const Schedule& sc = *j.sched;
      c.type = (const uint8_t*)put(nl.type.data(), nl.type.size());
      c.fi_off = (const uint32_t*)put(nl.fi_off.data(), nl.fi_off.size() * 4);
      c.fi_idx = (const uint32_t*)put(nl.fi_idx.data(), nl.fi_idx.size() * 4);
      c.level = (const uint32_t*)put(nl.level.data(), nl.level.size() * 4);
      c.lvl = (const uint4*)put(sc.lvl.data(), sc.lvl.size() * sizeof(LevelDesc));
      c.blob = (const uint4*)put(sc.blob.data(), sc.blob.size() * 8);
      c.li_off = (const uint32_t*)put(sc.li_off.data(), sc.li_off.size() * 4);
      c.li = (const uint32_t*)put(sc.li.data(), sc.li.size() * 4);
    }
    c.inj = (const InjRec*)put(p.sweeps.data(), p.sweeps.size() * sizeof(InjRec));
    c.roots = (const RootRec*)put(p.roots.data(), p.roots.size() * sizeof(RootRec));
    c.members = (const MemberRec*)put(p.members.data(), p.members.size() * sizeof(MemberRec));
    c.traced = (const TracedRec*)put(p.traced.data(), p.traced.size() * sizeof(TracedRec));
    c.traced_slot = (const uint32_t*)put(p.traced_slot.data(), p.traced_slot.size() * 4);
    c.exact_fault = (const uint32_t*)put(p.exact_fault.data(), p.exact_fault.size() * 4);
    c.pwords = j.good_resident ? nullptr : (const uint64_t*)put(j.pats->words.data(), j.pats->words.size() * 8);
  }
  if (at) CK(cudaMemcpyAsync(d_static.p, h_static.p, at, cudaMemcpyHostToDevice, s));
  static_bytes = at;
  return at;
}

void BatchExec::layout(const std::vector<BatchJob>& jobs, const std::vector<ClassShape>& shapes,
                       bool first_tile_only, cudaStream_t s) {
  invalidate_graph();
  tile0 = first_tile_only;
  const size_t n = jobs.size();
  circs.assign(n, BatchCirc{});
  res_off.assign(n, 0);
  F_total = 0;
  fault_patterns = 0;
  dense_gate_words = 0;
  sweep_alg_bytes = 0;
  good_gate_words = 0;

  // Sizes of every block (the ones batch_wave_bytes reports: a caller that
  // sized the buffers by it never sees them reallocated).
  const WaveBytes wb_need = batch_wave_bytes(jobs, first_tile_only);
  // Static arrays not resident on the device: one block, 256-byte aligned.
  d_static.ensure(wb_need.stat);
  h_static.ensure(wb_need.stat);
  upload_static(jobs, s);

  // Work arena (good, sweep outputs, sensitivities) and per-fault results.
  d_work.ensure(wb_need.work);
  for (const BatchJob& j : jobs) F_total += j.F;
  d_res.ensure(wb_need.res);
  {
    char* wb = d_work.as<char>();
    uint64_t at = 0;
    auto take = [&](uint64_t bytes) {
      char* p = wb + at;
      at += align256(bytes);
      return p;
    };
    uint64_t fo = 0;
    for (size_t i = 0; i < n; ++i) {
      const BatchJob& j = jobs[i];
      const Plan& p = *j.plan;
      BatchCirc& c = circs[i];
      const uint64_t W = j.pats->W;
      const uint32_t tiles_all = (uint32_t)std::max<uint64_t>(1, (W + kTileWords - 1) / kTileWords);
      const uint32_t tiles = first_tile_only ? 1 : tiles_all;
      c.P = j.pats->P;
      c.N = p.N;
      c.n_pi = p.n_pi;
      c.W = (uint32_t)W;
      c.tiles = tiles;
      c.n_sweeps = (uint32_t)p.sweeps.size();
      c.n_stem_sweeps = p.n_stem_sweeps;
      c.n_roots = (uint32_t)p.roots.size();
      c.n_exact = (uint32_t)p.exact_fault.size();
      c.max_gate_level = p.max_gate_level;
      c.n_levels = p.n_levels;
      c.n_slots = (uint32_t)(p.members.size() + p.roots.size());
      c.good = j.good_resident ? j.dev.good : (uint64_t*)take((uint64_t)tiles * p.N * kTileWords * 8);
      c.out = (uint64_t*)take((uint64_t)tiles * std::max<uint32_t>(c.n_sweeps, 1) * kTileWords * 8);
      c.sens = first_tile_only ? nullptr
                               : (uint64_t*)take((uint64_t)tiles * std::max<uint32_t>(c.n_slots, 1) * kTileWords * 8);
      res_off[i] = fo;
      fo += j.F;
      fault_patterns += j.F * j.pats->P;
      dense_gate_words += p.dense_sweep_gates * kTileWords * tiles;
      sweep_alg_bytes += p.dense_sweep_bytes * kTileWords * tiles;
      good_gate_words += (uint64_t)(p.N - p.n_pi) * kTileWords * tiles;
    }
    char* rb = d_res.as<char>();
    const uint64_t Fp = std::max<uint64_t>(F_total, 1);
    d_count = (unsigned long long*)rb;
    d_first = (unsigned long long*)(rb + Fp * 8);
    d_lastflag = (uint8_t*)(rb + Fp * 16);
    for (size_t i = 0; i < n; ++i) {
      circs[i].count = d_count + res_off[i];
      circs[i].first = d_first + res_off[i];
      circs[i].lastflag = d_lastflag + res_off[i];
    }
  }

  // Launch tables.
  // Good machine: per level index, segments (circuit, element range).
  segs.clear();
  level_first_seg.clear();
  level_units.clear();
  uint32_t max_levels = 0;
  for (const BatchJob& j : jobs) max_levels = std::max(max_levels, j.nl->n_levels);
  good_units = 0;
  for (uint32_t l = 0; l < max_levels; ++l) {
    level_first_seg.push_back((uint32_t)segs.size());
    unsigned long long u = 0;
    for (size_t i = 0; i < n; ++i) {
      const Netlist& nl = *jobs[i].nl;
      if (jobs[i].good_resident || l >= nl.n_levels) continue;
      const uint32_t lo = nl.level_off[l], hi = nl.level_off[l + 1];
      if (hi <= lo) continue;
      segs.push_back(BatchGoodSeg{(uint32_t)i, lo, hi, 0, u});
      u += (unsigned long long)(hi - lo) * circs[i].tiles;
    }
    level_units.push_back(u);
    good_units += u;
  }
  level_first_seg.push_back((uint32_t)segs.size());

  // Sweep classes: shapes[c] runs the jobs with cls == c.
  classes.clear();
  uint32_t n_counters = 0;
  for (int a = 0; a < 4; ++a) smem_attr[a] = 0;
  for (size_t ci = 0; ci < shapes.size(); ++ci) {
    const ClassShape& sh = shapes[ci];
    SweepClass k;
    k.id = (int)ci;
    k.shape = sh;
    uint32_t max_live = 1, widest = 1;
    unsigned long long items = 0;
    for (size_t i = 0; i < n; ++i) {
      if (jobs[i].cls != (int)ci || circs[i].n_sweeps == 0) continue;
      if (jobs[i].M != sh.M) throw ArgError{"batch job's words per item differ from its class"};
      const unsigned long long ci_items =
          (unsigned long long)circs[i].tiles * circs[i].n_sweeps * (kTileWords / sh.M);
      if (ci_items >= 0xFFFFFFFFull)
        throw LimitError{"a batch circuit has 2^32 or more sweep items; run it on its own"};
      k.circ_ids.push_back((uint32_t)i);
      items += ci_items;
      k.work += (double)jobs[i].plan->dense_sweep_gates * circs[i].tiles;
      max_live = std::max(max_live, jobs[i].sched->max_live);
      widest = std::max(widest, jobs[i].sched->max_block16);
    }
    if (k.circ_ids.empty()) continue;
    k.n_items = items;
    k.max_live = max_live;
    k.widest = widest;
    k.queue_base = n_counters;
    n_counters += (uint32_t)k.circ_ids.size();
    size_class(k, sh);
    classes.push_back(std::move(k));
  }

  // FFR / exact units: (circuit, tile, root) and (circuit, tile, exact fault).
  ffr_prefix.assign(n + 1, 0);
  exact_prefix.assign(n + 1, 0);
  for (size_t i = 0; i < n; ++i) {
    ffr_prefix[i + 1] = ffr_prefix[i] + (unsigned long long)circs[i].tiles * circs[i].n_roots;
    exact_prefix[i + 1] = exact_prefix[i] + (unsigned long long)circs[i].tiles * circs[i].n_exact;
  }
  ffr_units = ffr_prefix[n];
  exact_units = exact_prefix[n];

  // Descriptor block: circuits, good segments, class tables, unit prefixes.
  d_desc.ensure(wb_need.desc);
  h_desc.ensure(wb_need.desc);
  {
    uint8_t* hb = h_desc.as<uint8_t>();
    char* db = d_desc.as<char>();
    uint64_t at = 0;
    auto put = [&](const void* src, uint64_t bytes) -> const void* {
      const uint64_t o = at;
      if (bytes) std::memcpy(hb + o, src, bytes);
      at = o + align256(bytes);
      return db + o;
    };
    dd_circs = (const BatchCirc*)put(circs.data(), n * sizeof(BatchCirc));
    dd_segs = (const BatchGoodSeg*)put(segs.data(), segs.size() * sizeof(BatchGoodSeg));
    dd_ffr_prefix = (const unsigned long long*)put(ffr_prefix.data(), (n + 1) * 8);
    dd_exact_prefix = (const unsigned long long*)put(exact_prefix.data(), (n + 1) * 8);
    CK(cudaMemcpyAsync(d_desc.p, h_desc.p, at, cudaMemcpyHostToDevice, s));
    desc_bytes = at;
  }
  // Control words: one work counter per class and the error flag.
  ctl_bytes = align256(((uint64_t)n_counters + 1) * 8);
  d_ctl.ensure(wb_need.ctl);
  h_res.ensure(wb_need.res);
  n_circ = (uint32_t)n;
  // Host staging must outlive the copies above.
  CK(cudaStreamSynchronize(s));
}

void BatchExec::size_class(SweepClass& k, const ClassShape& sh) {
  k.shape = sh;
  const size_t share = sweep_smem_share(smem_optin, smem_per_sm, sh.occ);
  k.vals_bytes = sweep_vals_bytes(k.max_live, sh.M);
  if (k.vals_bytes > share)
    throw LimitError{"a batch circuit needs " + std::to_string(k.max_live) + " live values at " +
                     std::to_string(sh.M) + " word(s) per item; " + std::to_string(sh.occ) +
                     " CTA(s) per SM leave room for " + std::to_string(share / (8 * sh.M))};
  k.rec_buf = (uint32_t)std::min<size_t>(k.widest, (share - k.vals_bytes) / 32);
  k.smem = std::max<size_t>(16, k.vals_bytes + (size_t)k.rec_buf * 32);
  k.threads = std::min<int>(sh.threads, (int)sweep_max_threads(sh.M));
  size_t& attr = smem_attr[m_slot(sh.M)];
  attr = std::max(attr, k.smem);
  CK(sweep_batch_set_smem(sh.M, attr));
  int occ = 0;
  CK(sweep_batch_occupancy(sh.M, k.threads, k.smem, &occ));
  if (occ < 1) throw LimitError{"batch sweep kernel does not fit on an SM with this shape"};
  k.blocks = (int)std::min<unsigned long long>((unsigned long long)n_sms * occ, k.n_items);
}

void BatchExec::relaunch_shapes(const std::vector<ClassShape>& shapes) {
  // Same circuits and classes (same words per item); new CTA size / CTAs per SM.
  for (SweepClass& k : classes) {
    const ClassShape& sh = shapes[k.id];
    if (sh.M != k.shape.M) throw ArgError{"a class's words per item cannot change without a new layout"};
    size_class(k, sh);
  }
  invalidate_graph();
}

void BatchExec::apply_attributes() {
  for (int M : {1, 2, 4, 8})
    if (smem_attr[m_slot(M)]) CK(sweep_batch_set_smem(M, smem_attr[m_slot(M)]));
}

uint64_t BatchExec::enqueue(cudaStream_t s, bool good_only, bool with_events, cudaEvent_t* ev) {
  uint64_t launches = 0;
  CK(cudaMemsetAsync(d_ctl.p, 0, ctl_bytes, s));
  if (!tile0 && !good_only) {
    launch_init_results_batch(d_count, d_first, d_lastflag, F_total, s);
    launches += F_total ? 1 : 0;
  }
  for (size_t l = 0; l + 1 < level_first_seg.size(); ++l) {
    const uint32_t s0 = level_first_seg[l], s1 = level_first_seg[l + 1];
    if (s1 == s0) continue;
    launch_good_batch(dd_circs, dd_segs + s0, s1 - s0, level_units[l], s);
    ++launches;
  }
  CK(cudaGetLastError());
  if (with_events) CK(cudaEventRecord(ev[0], s));
  if (good_only) return launches;
  if (concurrent && classes.size() > 1) {
    launches += enqueue_sweeps_concurrent(s, with_events ? class_events : nullptr);
  } else if (with_events && class_events) {
    for (size_t ci = 0; ci < classes.size(); ++ci) {
      launches += enqueue_sweeps(s, classes[ci].id);
      CK(cudaEventRecord(class_events[ci], s));
    }
  } else {
    launches += enqueue_sweeps(s);
  }
  if (with_events) CK(cudaEventRecord(ev[1], s));
  if (!tile0) {
    BatchUnits u{dd_circs, dd_ffr_prefix, n_circ};
    launch_ffr_batch(u, ffr_units, s);
    launches += ffr_units ? 1 : 0;
    BatchUnits x{dd_circs, dd_exact_prefix, n_circ};
    launch_exact_batch(x, exact_units, s);
    launches += exact_units ? 1 : 0;
    CK(cudaGetLastError());
  }
  return launches;
}

uint64_t BatchExec::enqueue_sweeps_concurrent(cudaStream_t s, cudaEvent_t* class_end) {
  // One branch per class (up to kMaxBranches streams, then round-robin),
  // largest class first, forked from and joined back into s.
  constexpr size_t kMaxBranches = 32;
  const size_t nb = std::min(classes.size(), kMaxBranches);
  while (branch.size() < nb) {
    cudaStream_t x;
    CK(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    branch.push_back(x);
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    branch_done.push_back(e);
  }
  if (!fork_ev) CK(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
  std::vector<size_t> order(classes.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t a, size_t b) { return classes[a].work > classes[b].work; });
  CK(cudaEventRecord(fork_ev, s));
  for (size_t b = 0; b < nb; ++b) CK(cudaStreamWaitEvent(branch[b], fork_ev, 0));
  uint64_t launches = 0;
  for (size_t r = 0; r < order.size(); ++r) {
    const size_t ci = order[r];
    cudaStream_t x = branch[r % nb];
    launches += enqueue_sweeps(x, classes[ci].id);
    if (class_end) CK(cudaEventRecord(class_end[ci], x));
  }
  for (size_t b = 0; b < nb; ++b) {
    CK(cudaEventRecord(branch_done[b], branch[b]));
    CK(cudaStreamWaitEvent(s, branch_done[b], 0));
  }
  return launches;
}

uint64_t BatchExec::enqueue_sweeps(cudaStream_t s, int only) {
  uint64_t launches = 0;
  for (size_t ci = 0; ci < classes.size(); ++ci) {
    const SweepClass& k = classes[ci];
    if (only >= 0 && k.id != only) continue;
    // one launch per kSweepCircsPerLaunch circuits of the class
    for (size_t j0 = 0; j0 < k.circ_ids.size(); j0 += kSweepCircsPerLaunch) {
      const size_t j1 = std::min(k.circ_ids.size(), j0 + (size_t)kSweepCircsPerLaunch);
      params.n_circ = (uint32_t)(j1 - j0);
      unsigned long long chunk_items = 0;
      for (size_t j = j0; j < j1; ++j) {
        const BatchCirc& c = circs[k.circ_ids[j]];
        SweepCirc& d = params.c[j - j0];
        d.blob = c.blob;
        d.level = c.level;
        d.lvl = c.lvl;
        d.li_off = c.li_off;
        d.li = c.li;
        d.fi_off = c.fi_off;
        d.fi_idx = c.fi_idx;
        d.type = c.type;
        d.inj = c.inj;
        d.good = c.good;
        d.out = c.out;
        d.N = c.N;
        d.n_sweeps = c.n_sweeps;
        d.max_gate_level = c.max_gate_level;
        d.n_items = c.tiles * c.n_sweeps * (kTileWords / (uint32_t)k.shape.M);
        chunk_items += d.n_items;
      }
      params.queue = d_ctl.as<unsigned long long>() + 1 + k.queue_base + j0;
      params.err = d_ctl.as<int>();
      params.wait_ns = kWaitLimitNs;
      params.vals_bytes = k.vals_bytes;
      params.rec_buf = k.rec_buf;
      const int blocks = (int)std::min<unsigned long long>((unsigned long long)k.blocks, chunk_items);
      CK(launch_sweep_batch(k.shape.M, k.threads, std::max(blocks, 1), k.smem, params, s));
      ++launches;
    }
  }
  return launches;
}

void BatchExec::invalidate_graph() {
  if (gexec) cudaGraphExecDestroy(gexec);
  if (graph) cudaGraphDestroy(graph);
  gexec = nullptr;
  graph = nullptr;
}

uint64_t BatchExec::run_graph(cudaStream_t capture_stream, cudaStream_t s) {
  if (!gexec) {
    CK(cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeThreadLocal));
    try {
      graph_launches = enqueue(capture_stream, false, false, nullptr);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(capture_stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CK(cudaStreamEndCapture(capture_stream, &graph));
    CK(cudaGraphInstantiate(&gexec, graph, 0));
  }
  CK(cudaGraphLaunch(gexec, s));
  return graph_launches;
}

void BatchExec::fetch(cudaStream_t s, int* kerr) {
  const uint64_t Fp = std::max<uint64_t>(F_total, 1);
  char* hb = h_res.as<char>();
  if (F_total) {
    CK(cudaMemcpyAsync(hb, d_count, F_total * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hb + Fp * 8, d_first, F_total * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hb + Fp * 16, d_lastflag, F_total, cudaMemcpyDeviceToHost, s));
  }
  CK(cudaMemcpyAsync(hb + Fp * 17, d_ctl.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  std::memcpy(kerr, hb + Fp * 17, sizeof(int));
}

void BatchExec::results(size_t i, const BatchJob& j, fsimb_fault_result* out) const {
  const uint64_t Fp = std::max<uint64_t>(F_total, 1);
  const unsigned long long* cnt = (const unsigned long long*)h_res.p + res_off[i];
  const unsigned long long* fst = (const unsigned long long*)(h_res.as<char>() + Fp * 8) + res_off[i];
  const uint8_t* lf = (const uint8_t*)(h_res.as<char>() + Fp * 16) + res_off[i];
  const uint64_t W = j.pats->W;
  const uint64_t last_rd = W ? W - 1 : 0;
  for (uint64_t f = 0; f < j.F; ++f) {
    fsimb_fault_result& r = out[f];
    r = fsimb_fault_result{};
    r.count = cnt[f];
    r.detected = cnt[f] > 0;
    r.first_pattern = (fst[f] == ~0ull) ? -1 : (int64_t)fst[f];
    r.ref_last_round_flag = W ? lf[f] : 0;
    r.ref_last_rd = last_rd;
  }
}

uint64_t BatchExec::items() const {
  uint64_t s = 0;
  for (const SweepClass& k : classes) s += k.n_items;
  return s;
}

}  // namespace fsimb

// ------------------------------------------------------------ fsimb_batch

namespace {

struct MemberCache {
  uint64_t gen = 0;  // fsimb_handle::plan_gen the schedules belong to
  Schedule sched[4];
  bool has[4] = {false, false, false, false};
};

bool same_shapes(const std::vector<ClassShape>& a, const std::vector<ClassShape>& b) {
  if (a.size() != b.size()) return false;
  for (size_t i = 0; i < a.size(); ++i)
    if (a[i].M != b[i].M || a[i].threads != b[i].threads || a[i].occ != b[i].occ) return false;
  return true;
}

}  // namespace

// Words per item, class and class shapes of every member.
struct BatchAssign {
  std::vector<int> M, cls;
  std::vector<ClassShape> shapes;
  std::vector<uint32_t> max_live;  // per class: the largest member schedule's slots
};

struct fsimb_batch {
  int device = -1;
  int n_sms = 0;
  size_t smem_optin = 0, smem_per_sm = 0;
  cudaStream_t stream = nullptr;
  std::string err;

  std::vector<fsimb_handle*> members;
  std::vector<MemberCache> cache;

  BatchExec exec;
  // What the exec's layout was built from.
  std::vector<fsimb_handle*> laid_members;
  std::vector<uint64_t> laid_gens;
  std::vector<int> laid_M, laid_cls;
  std::vector<ClassShape> laid_shapes;
  bool laid = false;

  // Autotuner result for a membership (members and their generations).
  std::vector<fsimb_handle*> tuned_members;
  std::vector<uint64_t> tuned_gens;
  BatchAssign tuned;
  bool has_tuned = false;

  std::vector<cudaEvent_t> events;
  fsimb_batch_stats stats{};
  std::vector<double> class_ms;  // per class sweep time of the last direct-launch run

  cudaEvent_t ev(size_t i) {
    while (events.size() <= i) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      events.push_back(e);
    }
    return events[i];
  }

  ~fsimb_batch() {
    if (device >= 0) {
      cudaSetDevice(device);
      exec.release();
      for (auto e : events) cudaEventDestroy(e);
      if (stream) cudaStreamDestroy(stream);
    }
  }

  std::vector<uint64_t> gens() const {
    std::vector<uint64_t> g;
    for (const fsimb_handle* h : members) g.push_back(h->gen);
    return g;
  }

  // Plans for every member whose plan is stale; cached schedules of members
  // whose circuit or faults changed are dropped.
  void prepare_plans() {
    if (cache.size() != members.size()) cache.resize(members.size());
    for (size_t i = 0; i < members.size(); ++i) {
      fsimb_handle* h = members[i];
      if (!h->has_ckt || !h->has_faults || !h->has_pats)
        throw StateError{"batch member " + std::to_string(i) + " is not loaded (circuit, faults, patterns)"};
      if (cache[i].gen != h->plan_gen) {
        cache[i] = MemberCache{};
        cache[i].gen = h->plan_gen;
      }
    }
    parallel_for(members.size(), [&](size_t i) {
      fsimb_handle* h = members[i];
      if (!h->plan_valid) {
        build_plan(h->nl, h->faults, h->plan);
        h->plan_valid = true;
        h->plan_uploaded = false;
        h->sched_M = 0;
        h->sched_uploaded = false;
      }
    });
  }

  size_t smem_share(int occ) const { return sweep_smem_share(smem_optin, smem_per_sm, occ); }

  // Schedules for every member at words per item M or the largest smaller
  // value whose slots fit `share`; returns that value per member.
  std::vector<int> schedules(int M, size_t share) {
    std::vector<int> got(members.size(), 0);
    parallel_for(members.size(), [&](size_t i) {
      for (int m = M; m >= 1; m /= 2) {
        const Schedule& sc = schedule_at(i, m);
        if (sc.max_live <= kMaxSlots && sweep_vals_bytes(sc.max_live, m) <= share) {
          got[i] = m;
          return;
        }
      }
    });
    for (size_t i = 0; i < got.size(); ++i)
      if (!got[i])
        throw LimitError{"batch member " + std::to_string(i) +
                         " has more live values than shared memory holds at 1 word per item"};
    return got;
  }

  void level_widths(size_t i, std::vector<uint32_t>& widths) const {
    const Plan& p = members[i]->plan;
    for (uint32_t l = 1; l <= p.max_gate_level && l < p.n_levels; ++l)
      widths.push_back(p.level_off[l + 1] - p.level_off[l]);
  }

  // Automatic classes: each member at the default shape the plain path would
  // give it alone (default_sweep_shape, with the batch kernel's occupancy),
  // and members of the same shape share a class.  A class's shared memory is
  // capped at the share of its CTAs per SM, so no member runs at a lower
  // occupancy than alone.
  BatchAssign auto_assign() {
    BatchAssign a;
    const size_t n = members.size();
    a.M.resize(n);
    std::vector<ClassShape> shape(n);
    std::vector<long long> key(n);
    const size_t share2 = smem_share(2);
    parallel_for(n, [&](size_t i) {  // the schedules the default shape looks at first
      for (int m : {8, 4})
        if (sweep_vals_bytes(members[i]->plan.max_live, m) <= share2) schedule_at(i, m);
    });
    for (size_t i = 0; i < n; ++i) {
      std::vector<uint32_t> w;
      level_widths(i, w);
      uint32_t widest = 1;
      for (uint32_t x : w) widest = std::max(widest, x);
      int M = 0, occ = 1, t = 0;
      default_sweep_shape(
          members[i]->plan, [&](int m) -> const Schedule& { return schedule_at(i, m); },
          [&](int m, int th, size_t smem) {
            CK(sweep_batch_set_smem(m, smem));
            int got = 0;
            CK(sweep_batch_occupancy(m, th, smem, &got));
            return got;
          },
          std::move(w), widest, smem_optin, smem_per_sm, M, occ, t);
      if (sweep_vals_bytes(schedule_at(i, M).max_live, M) > smem_share(occ))
        throw LimitError{"batch member " + std::to_string(i) +
                         " has more live values than shared memory holds at 1 word per item"};
      a.M[i] = M;
      shape[i] = ClassShape{M, t, occ};
      key[i] = ((long long)m_slot(M) * 4096 + t) * 32 + occ;
    }
    std::vector<long long> keys(key);
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    a.cls.resize(n);
    a.shapes.resize(keys.size());
    a.max_live.assign(keys.size(), 0);
    for (size_t i = 0; i < n; ++i) {
      const int c = (int)(std::lower_bound(keys.begin(), keys.end(), key[i]) - keys.begin());
      a.cls[i] = c;
      a.shapes[c] = shape[i];
      a.max_live[c] = std::max(a.max_live[c], schedule_at(i, a.M[i]).max_live);
    }
    return a;
  }

  // The member's schedule at M words per item (built once per plan).
  const Schedule& schedule_at(size_t i, int m) {
    MemberCache& c = cache[i];
    const int sl = m_slot(m);
    if (!c.has[sl]) {
      build_schedule(members[i]->nl, members[i]->plan, 16u / (uint32_t)m, c.sched[sl]);
      c.has[sl] = true;
    }
    return c.sched[sl];
  }

  // Explicit shape: every member at words_per_item (or the largest smaller
  // value that fits), one class per words-per-item value.
  BatchAssign fixed_assign(int M, int threads, int occ) {
    BatchAssign a;
    a.M = schedules(M ? M : 8, smem_share(occ));
    a.cls.resize(members.size());
    for (int m : {8, 4, 2, 1}) {
      std::vector<uint32_t> w;
      bool any = false;
      for (size_t i = 0; i < members.size(); ++i)
        if (a.M[i] == m) {
          a.cls[i] = (int)a.shapes.size();
          level_widths(i, w);
          any = true;
        }
      if (!any) continue;
      a.shapes.push_back(ClassShape{m, threads ? threads : (int)pick_sweep_threads(w, m), occ});
    }
    return a;
  }

  std::vector<BatchJob> jobs_for(const std::vector<size_t>& idx, const BatchAssign& a) {
    std::vector<BatchJob> js(idx.size());
    for (size_t k = 0; k < idx.size(); ++k) {
      const size_t i = idx[k];
      fsimb_handle* h = members[i];
      BatchJob& j = js[k];
      j.nl = &h->nl;
      j.plan = &h->plan;
      j.pats = &h->pats;
      j.F = h->faults.size();
      j.M = a.M[i];
      j.cls = a.cls[i];
      j.sched = &cache[i].sched[m_slot(a.M[i])];
    }
    return js;
  }

  // Sweep time of class 0 of `tx` (work counters reset before each run):
  // the fastest of `runs` runs, after an untimed one when `warm`.
  float time_class0(BatchExec& tx, bool warm, cudaStream_t s, int runs) {
    cudaEvent_t e0 = ev(0), e1 = ev(1);
    float ms = 1e30f;
    for (int rep = warm ? -1 : 0; rep < runs; ++rep) {
      CK(cudaMemsetAsync(tx.d_ctl.p, 0, tx.ctl_bytes, s));
      CK(cudaEventRecord(e0, s));
      tx.enqueue_sweeps(s, 0);
      CK(cudaEventRecord(e1, s));
      CK(cudaEventSynchronize(e1));
      float x = 0;
      CK(cudaEventElapsedTime(&x, e0, e1));
      int kerr = 0;
      CK(cudaMemcpy(&kerr, tx.d_ctl.p, sizeof(int), cudaMemcpyDeviceToHost));
      if (kerr) throw CudaError{"a sweep kernel reached its wait limit during tuning"};
      if (rep >= 0) ms = std::min(ms, x);
    }
    return ms;
  }

  // Members that carry at least 1% of the batch's sweep work (the largest 64
  // at most) get a class of their own, tuned as the plain path tunes a
  // circuit alone over words per item x CTAs per SM x CTA size (256-1,024
  // threads), on strided samples of the first tile's sweeps: every
  // candidate once on about 256 sweeps, then the default and the three
  // fastest twice on about 1,024, the default kept unless beaten by 2%.  A shared class cannot give
  // each of these circuits its own shape, and they carry most of the work.
  // Returns, per class of the new assignment, whether its shape is final.
  std::vector<char> tune_singletons(BatchAssign& a, cudaStream_t s) {
    const size_t n = members.size();
    std::vector<double> wall(n);
    double total = 0;
    for (size_t i = 0; i < n; ++i) {
      const uint64_t tiles = std::max<uint64_t>(1, (members[i]->pats.W + kTileWords - 1) / kTileWords);
      wall[i] = ((double)members[i]->plan.dense_sweep_gates + 1.0) * (double)tiles;
      total += wall[i];
    }
    std::vector<size_t> dom;
    for (size_t i = 0; i < n; ++i)
      if (!members[i]->plan.sweeps.empty() && wall[i] >= 0.01 * total) dom.push_back(i);
    std::sort(dom.begin(), dom.end(), [&](size_t x, size_t y) { return wall[x] > wall[y]; });
    if (dom.size() > 64) dom.resize(64);
    if (dom.empty()) return std::vector<char>(a.shapes.size(), 0);

    std::vector<ClassShape> chosen(dom.size());
    bool warm = true;
    for (size_t d = 0; d < dom.size(); ++d) {
      const size_t i = dom[d];
      const Plan& P = members[i]->plan;
      const uint32_t ns = (uint32_t)P.sweeps.size();
      // Two samples: every stride-th sweep, about 256 (coarse) and about
      // 1,024 (fine) of them (timing only).
      Plan coarse = P, fine = P;
      for (Plan* q : {&coarse, &fine}) {
        const uint32_t stride = std::max<uint32_t>(1, ns / (q == &coarse ? 256u : 1024u));
        q->sweeps.clear();
        for (uint32_t k = 0; k < ns; k += stride) q->sweeps.push_back(P.sweeps[k]);
      }
      const ClassShape def = a.shapes[a.cls[i]];
      const size_t share1 = smem_share(1);
      auto fits_M = [&](int M) {
        if (sweep_vals_bytes(P.max_live, M) > share1) return false;
        const Schedule& sc = schedule_at(i, M);
        return sc.max_live <= kMaxSlots && sweep_vals_bytes(sc.max_live, M) <= share1;
      };
      // A one-circuit layout of `plan` at M, with its first tile's good machine.
      auto lay = [&](BatchExec& tx, const Plan& plan, int M) {
        BatchJob j;
        j.nl = &members[i]->nl;
        j.plan = &plan;
        j.sched = &schedule_at(i, M);
        j.pats = &members[i]->pats;
        j.F = members[i]->faults.size();
        j.M = M;
        j.cls = 0;
        tx.n_sms = n_sms;
        tx.smem_optin = smem_optin;
        tx.smem_per_sm = smem_per_sm;
        tx.layout({j}, {ClassShape{M, 256, 1}}, true, s);
        tx.enqueue(s, true, false, nullptr);
      };
      // Sizes class 0 of tx at sh; false if the shape does not run as asked.
      auto usable = [&](BatchExec& tx, const ClassShape& sh) {
        if (sweep_vals_bytes(schedule_at(i, sh.M).max_live, sh.M) > smem_share(sh.occ)) return false;
        SweepClass& kc = tx.classes[0];
        try {
          tx.size_class(kc, sh);
        } catch (const LimitError&) {
          return false;
        }
        if (sh.occ > 1 && kc.rec_buf < std::min<uint32_t>(kc.widest, 64)) return false;
        // fewer CTAs per SM than asked: the same as a smaller shape
        return kc.blocks >= (int)std::min<unsigned long long>((unsigned long long)n_sms * sh.occ, kc.n_items);
      };
      // Stage 1: every candidate once on the coarse sample.
      struct Timed {
        float ms;
        ClassShape sh;
      };
      std::vector<Timed> t1;
      for (int M : {8, 4, 2, 1}) {
        if (!fits_M(M)) continue;
        BatchExec tx;
        lay(tx, coarse, M);
        for (int occ : {1, 2, 3, 4})
          for (int T : {256, 384, 512, 768, 1024}) {
            const ClassShape sh{M, T, occ};
            if (T > (int)sweep_max_threads(M) || T * occ > 2048 || !usable(tx, sh)) continue;
            t1.push_back(Timed{time_class0(tx, warm, s, 1), sh});
            warm = false;
          }
        tx.release();
      }
      std::sort(t1.begin(), t1.end(), [](const Timed& x, const Timed& y) { return x.ms < y.ms; });
      // Stage 2: the default and the three fastest, twice each on the fine
      // sample; the default stays unless beaten by 2%.
      std::vector<ClassShape> fin{def};
      for (const Timed& t : t1) {
        if (fin.size() >= 4) break;
        if (!(t.sh.M == def.M && t.sh.occ == def.occ && t.sh.threads == def.threads)) fin.push_back(t.sh);
      }
      ClassShape best = def;
      float best_ms = 1e30f;
      bool best_is_default = false;
      for (int M : {8, 4, 2, 1}) {
        bool any = false;
        for (const ClassShape& sh : fin) any |= sh.M == M;
        if (!any || !fits_M(M)) continue;
        BatchExec tx;
        lay(tx, fine, M);
        for (const ClassShape& sh : fin) {
          if (sh.M != M || !usable(tx, sh)) continue;
          const float ms = time_class0(tx, warm, s, 2);
          warm = false;
          const bool is_default = sh.M == def.M && sh.occ == def.occ && sh.threads == def.threads;
          if (is_default || ms < (best_is_default ? 0.98f : 1.0f) * best_ms) {
            best_ms = ms;
            best = sh;
            best_is_default = is_default;
          }
        }
        tx.release();
      }
      chosen[d] = best;
    }

    // New assignment: the other members keep their shared classes, each
    // dominant member its own.
    std::vector<char> is_dom(n, 0);
    for (size_t i : dom) is_dom[i] = 1;
    BatchAssign b;
    b.M = a.M;
    b.cls.assign(n, -1);
    std::vector<int> remap(a.shapes.size(), -1);
    for (size_t i = 0; i < n; ++i) {
      if (is_dom[i]) continue;
      int& r = remap[a.cls[i]];
      if (r < 0) {
        r = (int)b.shapes.size();
        b.shapes.push_back(a.shapes[a.cls[i]]);
      }
      b.cls[i] = r;
    }
    std::vector<char> fixed(b.shapes.size(), 0);
    for (size_t d = 0; d < dom.size(); ++d) {
      b.cls[dom[d]] = (int)b.shapes.size();
      b.M[dom[d]] = chosen[d].M;
      b.shapes.push_back(chosen[d]);
      fixed.push_back(1);
    }
    b.max_live.assign(b.shapes.size(), 0);
    for (size_t i = 0; i < n; ++i)
      b.max_live[b.cls[i]] = std::max(b.max_live[b.cls[i]], schedule_at(i, b.M[i]).max_live);
    a = std::move(b);
    return fixed;
  }

  // Times candidate shapes per class (CTAs per SM x CTA size, words per item
  // fixed) on the first tile of a spread of the class's circuits (about 3%
  // of its sweep work); the default shape stays unless beaten by 2%.
  void autotune(BatchAssign& a, cudaStream_t s, const std::vector<char>& fixed) {
    const size_t n = members.size();
    const size_t n_cls = a.shapes.size();
    std::vector<double> w1(n), wall(n);
    for (size_t i = 0; i < n; ++i) {
      const uint64_t tiles = std::max<uint64_t>(1, (members[i]->pats.W + kTileWords - 1) / kTileWords);
      w1[i] = (double)members[i]->plan.dense_sweep_gates + 1.0;
      wall[i] = w1[i] * tiles;
    }
    std::vector<size_t> sample;
    for (size_t c = 0; c < n_cls; ++c) {
      if (fixed[c]) continue;  // tuned on its own already
      std::vector<size_t> in;
      double total = 0, t0 = 0;
      for (size_t i = 0; i < n; ++i)
        if (a.cls[i] == (int)c) {
          in.push_back(i);
          total += wall[i];
          t0 += w1[i];
        }
      std::sort(in.begin(), in.end(), [&](size_t x, size_t y) { return w1[x] < w1[y]; });
      const size_t k = std::max<size_t>(1, (size_t)(t0 / (0.03 * total)));
      size_t picked = 0;
      for (size_t q = k / 2; q < in.size(); q += k, ++picked) sample.push_back(in[q]);
      if (!picked && !in.empty()) sample.push_back(in.back());
    }
    std::sort(sample.begin(), sample.end());
    if (sample.empty()) return;

    BatchExec tx;
    tx.n_sms = n_sms;
    tx.smem_optin = smem_optin;
    tx.smem_per_sm = smem_per_sm;
    std::vector<BatchJob> js = jobs_for(sample, a);
    tx.layout(js, a.shapes, true, s);
    tx.enqueue(s, true, false, nullptr);  // good machine of the sampled tiles
    cudaEvent_t e0 = ev(0), e1 = ev(1);
    std::vector<ClassShape> cur = a.shapes;
    for (size_t c = 0; c < n_cls; ++c) {
      SweepClass* kc = nullptr;
      for (SweepClass& k : tx.classes)
        if (k.id == (int)c) kc = &k;
      if (!kc) continue;  // no sampled circuit in this class
      const ClassShape def = a.shapes[c];
      const int M = def.M;
      std::vector<ClassShape> cands{def};
      for (int occ : {1, 2, 3, 4})
        for (int T : {128, 256, 384, 512, 768, 1024})
          if (T <= (int)sweep_max_threads(M) && T * occ <= 2048 && !(occ == def.occ && T == def.threads))
            cands.push_back(ClassShape{M, T, occ});
      float best_ms = 1e30f;
      ClassShape best = def;
      bool best_is_default = false;
      for (const ClassShape& sh : cands) {
        // every member of the class, not only the sampled ones, must fit
        if (sweep_vals_bytes(a.max_live[c], M) > smem_share(sh.occ)) continue;
        try {
          tx.size_class(*kc, sh);
        } catch (const LimitError&) {
          continue;  // slots do not fit this many CTAs per SM
        }
        if (kc->blocks < (int)std::min<unsigned long long>((unsigned long long)n_sms * sh.occ, kc->n_items))
          continue;  // fewer CTAs per SM than asked: the same as a smaller shape
        // an untimed run of the first candidate warms the GPU up; then the
        // fastest of two timed runs counts
        float ms = 1e30f;
        for (int rep = (&sh == &cands[0]) ? -1 : 0; rep < 2; ++rep) {
          CK(cudaMemsetAsync(tx.d_ctl.p, 0, tx.ctl_bytes, s));
          CK(cudaEventRecord(e0, s));
          tx.enqueue_sweeps(s, (int)c);
          CK(cudaEventRecord(e1, s));
          CK(cudaEventSynchronize(e1));
          float x = 0;
          CK(cudaEventElapsedTime(&x, e0, e1));
          int kerr = 0;
          CK(cudaMemcpy(&kerr, tx.d_ctl.p, sizeof(int), cudaMemcpyDeviceToHost));
          if (kerr) throw CudaError{"a sweep kernel reached its wait limit during tuning"};
          if (rep >= 0) ms = std::min(ms, x);
        }
        // the default shape stays unless a candidate beats it by 2%
        const bool is_default = sh.occ == def.occ && sh.threads == def.threads;
        if (is_default || ms < (best_is_default ? 0.98f : 1.0f) * best_ms) {
          best_ms = ms;
          best = sh;
          best_is_default = is_default;
        }
      }
      tx.size_class(*kc, best);
      cur[c] = best;
    }
    a.shapes = cur;
    tx.release();
  }

  void run(const fsimb_batch_opts* opts);
};

void fsimb_batch::run(const fsimb_batch_opts* opts) {
  fsimb_batch_opts o{};
  if (opts) {
    if (opts->struct_size != 0 && opts->struct_size < sizeof(fsimb_batch_opts))
      throw ArgError{"fsimb_batch_opts.struct_size too small"};
    o = *opts;
  }
  if (o.words_per_item && o.words_per_item != 1 && o.words_per_item != 2 && o.words_per_item != 4 &&
      o.words_per_item != 8)
    throw ArgError{"words_per_item must be 0, 1, 2, 4 or 8"};
  if (o.block_threads && (o.block_threads < 32 || o.block_threads > 1024 || o.block_threads % 32))
    throw ArgError{"block_threads must be 0 or a multiple of 32 in 32..1024"};
  if (o.ctas_per_sm > 4) throw ArgError{"ctas_per_sm must be 0..4"};
  if (members.empty()) throw StateError{"the batch has no members"};
  CK(cudaSetDevice(device));
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : stream;
  for (fsimb_handle* h : members) h->has_results = false;

  const auto host0 = std::chrono::steady_clock::now();
  prepare_plans();
  const std::vector<uint64_t> g = gens();
  std::vector<size_t> all(members.size());
  for (size_t i = 0; i < all.size(); ++i) all[i] = i;

  // Classes and shapes: explicit options, the tuned shapes of this
  // membership, or the automatic classes.
  double tune_ms = 0;
  BatchAssign a;
  const bool explicit_shape = o.words_per_item || o.block_threads || o.ctas_per_sm;
  if (explicit_shape) {
    a = fixed_assign((int)o.words_per_item, (int)o.block_threads, o.ctas_per_sm ? (int)o.ctas_per_sm : 1);
  } else if (o.tune) {
    if (!has_tuned || tuned_members != members || tuned_gens != g) {
      const auto t0 = std::chrono::steady_clock::now();
      tuned = auto_assign();
      const std::vector<char> fixed = tune_singletons(tuned, s);
      autotune(tuned, s, fixed);
      tuned_members = members;
      tuned_gens = g;
      has_tuned = true;
      tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    a = tuned;
  } else {
    a = auto_assign();
  }
  const bool relayout = !laid || laid_members != members || laid_gens != g || laid_M != a.M ||
                        laid_cls != a.cls || !same_shapes(laid_shapes, a.shapes);
  const double host_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - host0).count() - tune_ms;

  cudaEvent_t e0 = ev(2), e1 = ev(3), e2 = ev(4), e3 = ev(5), p0 = ev(6), p1 = ev(7);
  CK(cudaEventRecord(e0, s));
  uint64_t h2d = 0;
  if (relayout) {
    laid = false;
    exec.layout(jobs_for(all, a), a.shapes, false, s);
    h2d = exec.static_bytes + exec.desc_bytes;
    laid_members = members;
    laid_gens = g;
    laid_M = a.M;
    laid_cls = a.cls;
    laid_shapes = a.shapes;
    laid = true;
  } else if (o.reupload) {
    h2d = exec.upload_static(jobs_for(all, a), s);
  }
  CK(cudaEventRecord(e1, s));
  uint64_t launches = 0;
  const bool graph = !o.no_graph;
  if (exec.concurrent != !o.serial_classes) {
    exec.concurrent = !o.serial_classes;
    exec.invalidate_graph();
  }
  exec.apply_attributes();  // the autotuner may have changed them
  if (graph) {
    launches = exec.run_graph(stream, s);
  } else {
    cudaEvent_t pe[2] = {p0, p1};
    std::vector<cudaEvent_t> ce;
    for (size_t ci = 0; ci < exec.classes.size(); ++ci) ce.push_back(ev(8 + ci));
    exec.class_events = ce.data();
    launches = exec.enqueue(s, false, true, pe);
    exec.class_events = nullptr;
  }
  CK(cudaEventRecord(e2, s));
  int kerr = 0;
  exec.fetch(s, &kerr);
  CK(cudaEventRecord(e3, s));
  CK(cudaEventSynchronize(e3));
  if (kerr) throw CudaError{"a sweep kernel reached its wait limit for a record copy; results discarded"};

  const std::vector<BatchJob> js = jobs_for(all, a);
  for (size_t i = 0; i < members.size(); ++i) {
    fsimb_handle* h = members[i];
    h->results.resize(js[i].F);
    exec.results(i, js[i], h->results.data());
    h->has_results = true;
  }

  stats = fsimb_batch_stats{};
  float x = 0;
  CK(cudaEventElapsedTime(&x, e0, e3));
  stats.ms_total = x;
  CK(cudaEventElapsedTime(&x, e0, e1));
  stats.ms_h2d = x;
  CK(cudaEventElapsedTime(&x, e1, e2));
  stats.ms_compute = x;
  CK(cudaEventElapsedTime(&x, e2, e3));
  stats.ms_d2h = x;
  class_ms.assign(exec.classes.size(), 0.0);
  if (!graph) {
    for (size_t ci = 0; ci < exec.classes.size(); ++ci) {
      // concurrent classes: from the end of the good machine to the class's end
      CK(cudaEventElapsedTime(&x, (exec.concurrent || !ci) ? p0 : ev(8 + ci - 1), ev(8 + ci)));
      class_ms[ci] = x;
    }
    CK(cudaEventElapsedTime(&x, e1, p0));
    stats.ms_good = x;
    CK(cudaEventElapsedTime(&x, p0, p1));
    stats.ms_sweep = x;
    CK(cudaEventElapsedTime(&x, p1, e2));
    stats.ms_ffr = x;
  }
  stats.ms_tune = tune_ms;
  stats.ms_host_prep = host_ms;
  stats.n_circuits = members.size();
  stats.n_faults = exec.F_total;
  stats.fault_patterns = exec.fault_patterns;
  stats.sweep_items = exec.items();
  stats.ffr_units = exec.ffr_units;
  stats.exact_units = exec.exact_units;
  stats.good_units = exec.good_units;
  stats.dense_gate_words = exec.dense_gate_words;
  stats.sweep_alg_bytes = exec.sweep_alg_bytes;
  stats.good_gate_words = exec.good_gate_words;
  stats.kernel_launches = launches;
  stats.graph_used = graph ? 1 : 0;
  stats.n_classes = (uint32_t)exec.classes.size();
  if (!exec.classes.empty()) {
    const SweepClass* big = &exec.classes[0];
    for (const SweepClass& k : exec.classes)
      if (k.n_items > big->n_items) big = &k;
    stats.words_per_item = (uint32_t)big->shape.M;
    stats.block_threads = (uint32_t)big->threads;
    stats.blocks = (uint32_t)big->blocks;
    stats.smem_bytes = (uint32_t)big->smem;
    stats.ctas_per_sm = (uint32_t)(big->blocks / std::max(1, n_sms));
  }
  stats.device_bytes = exec.device_bytes();
  stats.h2d_bytes = h2d;
  stats.d2h_bytes = exec.F_total * 17 + sizeof(int);
}

// -------------------------------------------------------------------- C ABI
extern "C" {

static thread_local std::string g_batch_create_error;

int fsimb_batch_create(int device, fsimb_batch** out) {
  if (!out) return FSIMB_ERR_ARG;
  *out = nullptr;
  fsimb_batch* b = nullptr;
  try {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || device < 0 || device >= n) {
      cudaGetLastError();
      g_batch_create_error = std::string("no usable CUDA device ") + std::to_string(device);
      return FSIMB_ERR_CUDA;
    }
    b = new fsimb_batch();
    b->device = device;
    CK(cudaSetDevice(device));
    int v = 0;
    CK(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
    b->n_sms = v;
    CK(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    b->smem_optin = (size_t)v;
    CK(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device));
    b->smem_per_sm = (size_t)v;
    CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->exec.n_sms = b->n_sms;
    b->exec.smem_optin = b->smem_optin;
    b->exec.smem_per_sm = b->smem_per_sm;
    *out = b;
    return FSIMB_OK;
  } catch (const CudaError& e) {
    g_batch_create_error = e.msg;
    delete b;
    return FSIMB_ERR_CUDA;
  } catch (const std::bad_alloc&) {
    g_batch_create_error = "host allocation failed";
    delete b;
    return FSIMB_ERR_NOMEM;
  }
}

int fsimb_batch_destroy(fsimb_batch* b) {
  delete b;
  return FSIMB_OK;
}

const char* fsimb_batch_last_error(const fsimb_batch* b) {
  return b ? b->err.c_str() : g_batch_create_error.c_str();
}

int fsimb_batch_add(fsimb_batch* b, fsimb_handle* h) {
  API_BEGIN(b)
  if (!h) throw ArgError{"null member handle"};
  if (std::find(b->members.begin(), b->members.end(), h) != b->members.end())
    throw ArgError{"handle is already a member of this batch"};
  b->members.push_back(h);
  API_END(b)
}

int fsimb_batch_clear(fsimb_batch* b) {
  API_BEGIN(b)
  b->members.clear();
  b->cache.clear();
  API_END(b)
}

int fsimb_batch_size(const fsimb_batch* b, uint64_t* n) {
  if (!b || !n) return FSIMB_ERR_ARG;
  *n = b->members.size();
  return FSIMB_OK;
}

int fsimb_batch_run(fsimb_batch* b, const fsimb_batch_opts* opts) {
  API_BEGIN(b)
  b->run(opts);
  API_END(b)
}

int fsimb_batch_class_stats(const fsimb_batch* b, uint32_t i, fsimb_batch_class* out) {
  if (!b || !out) return FSIMB_ERR_ARG;
  if (i >= b->exec.classes.size()) return FSIMB_ERR_ARG;
  const SweepClass& k = b->exec.classes[i];
  *out = fsimb_batch_class{};
  out->words_per_item = (uint32_t)k.shape.M;
  out->block_threads = (uint32_t)k.threads;
  out->blocks = (uint32_t)k.blocks;
  out->smem_bytes = (uint32_t)k.smem;
  out->n_circuits = k.circ_ids.size();
  out->sweep_items = k.n_items;
  out->max_live = k.max_live;
  out->widest_level = k.widest;
  out->ms_sweep = i < b->class_ms.size() ? b->class_ms[i] : 0.0;
  return FSIMB_OK;
}

int fsimb_batch_class_members(const fsimb_batch* b, uint32_t i, uint32_t* out, uint64_t n) {
  if (!b) return FSIMB_ERR_ARG;
  if (i >= b->exec.classes.size()) return FSIMB_ERR_ARG;
  const SweepClass& k = b->exec.classes[i];
  if (n < k.circ_ids.size() || (!out && !k.circ_ids.empty())) return FSIMB_ERR_ARG;
  std::copy(k.circ_ids.begin(), k.circ_ids.end(), out);
  return FSIMB_OK;
}

int fsimb_batch_get_stats(const fsimb_batch* b, fsimb_batch_stats* out) {
  if (!b || !out) return FSIMB_ERR_ARG;
  *out = b->stats;
  return FSIMB_OK;
}

}  // extern "C"
