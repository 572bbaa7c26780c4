// Serving loop (fsimb_server_* of include/fsimb.h): fault-simulation requests
// against resident circuits, admitted by device footprint and run in waves
// on a few concurrent slots.
//
//   * A resident circuit keeps on the device its CSR, its sweep schedule and
//     a block of patterns with the good-machine values of that block, so a
//     request names a fault subset and a range of the block's rows and
//     neither uploads the circuit nor re-runs the good machine.  A request
//     may also bring its own patterns; its good machine then runs in its
//     wave.
//   * Submitting is thread-safe and returns a ticket at once.  Planner
//     threads build each request's fault plan (build_fault_plan: O(faults +
//     touched FFR members)) and its exact device footprint.
//   * Each slot owns fixed device and pinned buffers, allocated once when the
//     server starts, so serving allocates nothing.  A dispatcher thread forms
//     a wave from planned requests in ticket order while the wave fits the
//     free slot's buffers, lays it out and launches it (the batch kernels),
//     queues the result copies and a host callback, and moves on: while one
//     slot's wave runs, requests that arrive are planned and launched on the
//     next free slot, and the waves overlap on the GPU.
//   * A request's results are the ones fsimb_run gives for the same circuit,
//     faults and patterns: the same kernels on the same data.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/fsimb.h"
#include "fsimb_batch.h"
#include "fsimb_internal.h"
#include "fsimb_kernels.cuh"

using namespace fsimb;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

int m_slot_s(int M) { return M == 1 ? 0 : M == 2 ? 1 : M == 4 ? 2 : 3; }

struct ResidentCircuit {
  Netlist nl;
  CircuitPlan cp;
  Schedule sched;
  ClassShape shape{4, 256, 1};
  Patterns block;  // resident pattern block (host copy of its words)
  uint64_t block_tiles = 0;
  // d_level_off holds the schedule's level descriptors, d_recs its record blocks
  DevBuf d_type, d_fi_off, d_fi_idx, d_level, d_level_off, d_recs, d_li_off, d_li, d_pwords, d_good;
  BatchCirc dev{};
  uint64_t device_bytes() const {
    uint64_t s = 0;
    for (const DevBuf* b : {&d_type, &d_fi_off, &d_fi_idx, &d_level, &d_level_off, &d_recs, &d_li_off,
                            &d_li, &d_pwords, &d_good})
      s += b->n;
    return s;
  }
  void release() {
    for (DevBuf* b : {&d_type, &d_fi_off, &d_fi_idx, &d_level, &d_level_off, &d_recs, &d_li_off, &d_li,
                      &d_pwords, &d_good})
      b->release();
  }
};

struct Request {
  uint64_t ticket = 0;
  uint32_t circuit = 0;
  std::vector<Fault> faults;
  Patterns pats;  // W and P; words only for a request with its own patterns
  bool own_patterns = false;
  uint64_t row0 = 0;
  Plan plan;
  BatchJob job;
  WaveBytes bytes;
  double work = 0;  // gate-word evaluations of its sweeps (the wave-time predictor)
  std::vector<fsimb_fault_result> results;
  int status = FSIMB_OK;
  std::string error;
  bool done = false;
  Clock::time_point t_submit, t_planned, t_launch, t_done;
};

struct Slot {
  BatchExec exec;
  cudaStream_t stream = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  WaveBytes cap;
  std::vector<Request*> wave;
  std::vector<BatchJob> jobs;
  bool busy = false;
  std::atomic<bool> finished{false};
  struct fsimb_server* owner = nullptr;
};

}  // namespace

struct fsimb_server {
  int device = -1;
  int n_sms = 0;
  size_t smem_optin = 0, smem_per_sm = 0;
  std::string err;
  fsimb_server_opts opts{};

  std::mutex circuits_mu;  // guards `circuits` growth
  // Held while kernel attributes are set and the launches that rely on them
  // are issued (circuit registration queries occupancy with its own sizes).
  std::mutex attr_mu;
  std::vector<std::unique_ptr<ResidentCircuit>> circuits;

  std::mutex mu;  // guards everything below
  std::condition_variable work_cv;  // planners and dispatcher wait here
  std::condition_variable done_cv;  // fsimb_server_wait waits here
  bool stopping = false;
  uint64_t next_ticket = 1;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
  std::deque<Request*> to_plan;
  std::map<uint64_t, Request*> ready;  // planned, by ticket
  uint64_t planning = 0;               // requests being planned

  std::vector<std::unique_ptr<Slot>> slots;
  std::vector<std::thread> planners;
  std::thread dispatcher;

  // statistics since the last reset
  std::vector<double> lat_ms, queue_ms, gpu_ms;
  uint64_t stat_completed = 0, stat_failed = 0, stat_waves = 0, stat_wave_requests = 0;
  double stat_fault_patterns = 0;
  bool stat_any = false;
  Clock::time_point stat_first_submit, stat_last_done;
  double stat_busy_ms = 0;
  // Gate-word evaluations per ms of waves so far (exponential average); it
  // turns a request's work into a predicted wave time.
  double gwe_per_ms = 3e8;

  ~fsimb_server() { shutdown(); }

  void shutdown() {
    {
      std::lock_guard<std::mutex> g(mu);
      if (stopping && !dispatcher.joinable()) return;
      stopping = true;
    }
    work_cv.notify_all();
    for (auto& t : planners)
      if (t.joinable()) t.join();
    if (dispatcher.joinable()) dispatcher.join();
    if (device >= 0) {
      cudaSetDevice(device);
      for (auto& s : slots) {
        if (s->stream) cudaStreamSynchronize(s->stream);
        s->exec.release();
        if (s->e0) cudaEventDestroy(s->e0);
        if (s->e1) cudaEventDestroy(s->e1);
        if (s->stream) cudaStreamDestroy(s->stream);
      }
      for (auto& c : circuits) c->release();
    }
    slots.clear();
  }

  static WaveBytes overhead() {  // a wave's sizes beyond the sum of its requests' shares
    WaveBytes w;
    w.res = 1024;
    w.desc = 2048;
    w.ctl = 512;
    return w;
  }

  static bool fits(const WaveBytes& need, const WaveBytes& cap) {
    return need.stat <= cap.stat && need.work <= cap.work && need.res <= cap.res &&
           need.desc <= cap.desc && need.ctl <= cap.ctl;
  }

  static void add(WaveBytes& a, const WaveBytes& b) {
    a.stat += b.stat;
    a.work += b.work;
    a.res += b.res;
    a.desc += b.desc;
    a.ctl += b.ctl;
  }

  void start() {
    const uint32_t nslots = opts.slots ? opts.slots : 2;
    const uint64_t sb = opts.slot_bytes ? opts.slot_bytes : (4ull << 30);
    for (uint32_t i = 0; i < nslots; ++i) {
      auto s = std::make_unique<Slot>();
      s->owner = this;
      CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
      CK(cudaEventCreate(&s->e0));
      CK(cudaEventCreate(&s->e1));
      s->exec.n_sms = n_sms;
      s->exec.smem_optin = smem_optin;
      s->exec.smem_per_sm = smem_per_sm;
      auto part = [&](double f) { return (uint64_t)(sb * f) / 256 * 256; };
      s->cap.work = part(0.72);
      s->cap.stat = part(0.12);
      s->cap.res = part(0.08);
      s->cap.desc = part(0.06);
      s->cap.ctl = std::max<uint64_t>(part(0.02), 4096);
      // every buffer at its final size now: serving allocates nothing
      s->exec.d_work.ensure(s->cap.work);
      s->exec.d_static.ensure(s->cap.stat);
      s->exec.d_res.ensure(s->cap.res);
      s->exec.d_desc.ensure(s->cap.desc);
      s->exec.d_ctl.ensure(s->cap.ctl);
      s->exec.h_static.ensure(s->cap.stat);
      s->exec.h_res.ensure(s->cap.res);
      s->exec.h_desc.ensure(s->cap.desc);
      slots.push_back(std::move(s));
    }
    const uint32_t np = opts.planner_threads
                            ? opts.planner_threads
                            : std::max(1u, std::min(8u, std::thread::hardware_concurrency() / 2));
    for (uint32_t i = 0; i < np; ++i) planners.emplace_back([this] { plan_loop(); });
    dispatcher = std::thread([this] { dispatch_loop(); });
  }

  ResidentCircuit& circuit(uint32_t id) {
    std::lock_guard<std::mutex> g(circuits_mu);
    if (id >= circuits.size()) throw ArgError{"unknown circuit id " + std::to_string(id)};
    return *circuits[id];
  }

  uint32_t add_circuit(const char* ckt, size_t len, const uint64_t* words, uint64_t n_patterns) {
    auto c = std::make_unique<ResidentCircuit>();
    bool loaded = false;
    if (len >= kDeviceLoadBytes) {  // large circuits: the device loader, on a stream of its own
      CK(cudaSetDevice(device));
      cudaStream_t ls;
      CK(cudaStreamCreateWithFlags(&ls, cudaStreamNonBlocking));
      LoadInfo li;
      try {
        loaded = parse_ckt_device(ckt, len, c->nl, device, ls, 0, li);
      } catch (const CudaError&) {
        loaded = false;  // no room on the device (or the like): the host reader still can
        cudaStreamSynchronize(ls);
        cudaGetLastError();
      } catch (...) {
        cudaStreamDestroy(ls);
        throw;
      }
      cudaStreamDestroy(ls);
    }
    if (!loaded) parse_ckt(ckt, len, c->nl);
    const Netlist& nl = c->nl;
    if (n_patterns && !words) throw ArgError{"null pattern words"};
    c->block.P = n_patterns;
    c->block.W = (n_patterns + 63) / 64;
    if (words) c->block.words.assign(words, words + c->block.W * nl.n_pi);
    build_circuit_plan(nl, c->cp);
    // the default shape, for the batch kernel
    std::vector<uint32_t> widths;
    uint32_t widest = 1;
    const Plan& B = c->cp.base;
    for (uint32_t l = 1; l <= B.max_gate_level && l < B.n_levels; ++l) {
      widths.push_back(B.level_off[l + 1] - B.level_off[l]);
      widest = std::max(widest, widths.back());
    }
    Schedule sc[4];
    bool has[4] = {false, false, false, false};
    auto sched_at = [&](int m) -> const Schedule& {
      const int sl = m_slot_s(m);
      if (!has[sl]) {
        build_schedule(nl, B, 16u / (uint32_t)m, sc[sl]);
        has[sl] = true;
      }
      return sc[sl];
    };
    // the schedules the default shape looks at first, before taking the lock
    for (int m : {8, 4})
      if (sweep_vals_bytes(B.max_live, m) <= sweep_smem_share(smem_optin, smem_per_sm, 2)) sched_at(m);
    int M = 0, occ = 1, T = 0;
    {
      std::lock_guard<std::mutex> g(attr_mu);
      default_sweep_shape(
          B, sched_at,
          [&](int m, int th, size_t smem) {
            CK(sweep_batch_set_smem(m, smem));
            int got = 0;
            CK(sweep_batch_occupancy(m, th, smem, &got));
            return got;
          },
          widths, widest, smem_optin, smem_per_sm, M, occ, T);
    }
    const Schedule& chosen = sched_at(M);
    if (chosen.max_live > kMaxSlots ||
        sweep_vals_bytes(chosen.max_live, M) > sweep_smem_share(smem_optin, smem_per_sm, occ))
      throw LimitError{"the circuit has more live values than shared memory holds at 1 word per item"};
    c->sched = chosen;
    c->shape = ClassShape{M, T, occ};

    // resident device data
    CK(cudaSetDevice(device));
    cudaStream_t s;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    try {
      upload(c->d_type, nl.type, s);
      upload(c->d_fi_off, nl.fi_off, s);
      upload(c->d_fi_idx, nl.fi_idx, s);
      upload(c->d_level, nl.level, s);
      upload(c->d_level_off, c->sched.lvl, s);
      upload(c->d_recs, c->sched.blob, s);
      upload(c->d_li_off, c->sched.li_off, s);
      upload(c->d_li, c->sched.li, s);
      c->block_tiles = (c->block.W + kTileWords - 1) / kTileWords;
      if (c->block.W) {
        upload(c->d_pwords, c->block.words, s);
        c->d_good.ensure(c->block_tiles * nl.N * kTileWords * 8);
        for (uint32_t l = 0; l < nl.n_levels; ++l) {
          GoodArgs g{};
          g.type = c->d_type.as<uint8_t>();
          g.fi_off = c->d_fi_off.as<uint32_t>();
          g.fi_idx = c->d_fi_idx.as<uint32_t>();
          g.pwords = c->d_pwords.as<uint64_t>();
          g.good = c->d_good.as<uint64_t>();
          g.n_pi = (uint32_t)nl.n_pi;
          g.N = nl.N;
          g.lo = nl.level_off[l];
          g.hi = nl.level_off[l + 1];
          g.W = (uint32_t)c->block.W;
          g.W_pad = (uint32_t)(c->block_tiles * kTileWords);
          launch_good_level(g, s);
        }
        CK(cudaGetLastError());
      }
      CK(cudaStreamSynchronize(s));
    } catch (...) {
      cudaStreamDestroy(s);
      c->release();
      throw;
    }
    CK(cudaStreamDestroy(s));
    c->dev.type = c->d_type.as<uint8_t>();
    c->dev.fi_off = c->d_fi_off.as<uint32_t>();
    c->dev.fi_idx = c->d_fi_idx.as<uint32_t>();
    c->dev.level = c->d_level.as<uint32_t>();
    c->dev.lvl = c->d_level_off.as<uint4>();
    c->dev.blob = c->d_recs.as<uint4>();
    c->dev.li_off = c->d_li_off.as<uint32_t>();
    c->dev.li = c->d_li.as<uint32_t>();
    std::lock_guard<std::mutex> g(circuits_mu);
    circuits.push_back(std::move(c));
    return (uint32_t)(circuits.size() - 1);
  }

  uint64_t submit(const fsimb_request& q) {
    ResidentCircuit& c = circuit(q.circuit);
    auto r = std::make_unique<Request>();
    r->circuit = q.circuit;
    if (q.n_faults && (!q.site || !q.value)) throw ArgError{"null fault arrays"};
    r->faults.resize(q.n_faults);
    for (uint64_t i = 0; i < q.n_faults; ++i) {
      if (q.site[i] >= c.nl.N) throw ArgError{"fault site out of range at " + std::to_string(i)};
      const uint8_t p = q.pin ? q.pin[i] : 0;
      if (p > c.nl.fanin_count(q.site[i])) throw ArgError{"fault pin out of range at " + std::to_string(i)};
      r->faults[i] = Fault{q.site[i], p, (uint8_t)(q.value[i] ? 1 : 0)};
    }
    r->pats.P = q.n_patterns;
    r->pats.W = (q.n_patterns + 63) / 64;
    if (q.words) {
      r->own_patterns = true;
      r->pats.words.assign(q.words, q.words + r->pats.W * c.nl.n_pi);
    } else {
      if (q.row0 % kTileWords) throw ArgError{"row0 must be a multiple of 32 (a 2,048-pattern tile)"};
      if (q.row0 + r->pats.W > c.block.W)
        throw ArgError{"rows " + std::to_string(q.row0) + ".." + std::to_string(q.row0 + r->pats.W) +
                       " exceed the circuit's resident block of " + std::to_string(c.block.W) + " rows"};
      r->row0 = q.row0;
    }
    r->t_submit = Clock::now();
    std::unique_lock<std::mutex> g(mu);
    if (stopping) throw StateError{"the server is shutting down"};
    r->ticket = next_ticket++;
    if (!stat_any) {
      stat_any = true;
      stat_first_submit = r->t_submit;
    }
    Request* raw = r.get();
    requests.emplace(raw->ticket, std::move(r));
    to_plan.push_back(raw);
    g.unlock();
    work_cv.notify_all();
    return raw->ticket;
  }

  void plan_loop() {
    for (;;) {
      Request* r = nullptr;
      {
        std::unique_lock<std::mutex> g(mu);
        work_cv.wait(g, [&] { return stopping || !to_plan.empty(); });
        if (to_plan.empty()) return;  // stopping
        r = to_plan.front();
        to_plan.pop_front();
        ++planning;
      }
      int status = FSIMB_OK;
      std::string msg;
      try {
        ResidentCircuit& c = circuit(r->circuit);
        build_fault_plan(c.nl, c.cp, r->faults, r->plan);
        BatchJob& j = r->job;
        j.nl = &c.nl;
        j.plan = &r->plan;
        j.sched = &c.sched;
        j.pats = &r->pats;
        j.F = r->faults.size();
        j.M = c.shape.M;
        j.resident = true;
        j.dev = c.dev;
        j.good_resident = !r->own_patterns;
        if (j.good_resident)
          j.dev.good = c.d_good.as<uint64_t>() + (r->row0 / kTileWords) * (uint64_t)c.nl.N * kTileWords;
        r->bytes = batch_job_bytes(j, false);
        r->work = (double)r->plan.dense_sweep_gates * kTileWords *
                  (double)std::max<uint64_t>(1, (r->pats.W + kTileWords - 1) / kTileWords);
        WaveBytes need = overhead();
        add(need, r->bytes);
        if (!slots.empty() && !fits(need, slots[0]->cap))
          throw LimitError{"the request needs more device memory than a slot holds"};
      } catch (const LimitError& e) {
        status = FSIMB_ERR_LIMIT;
        msg = e.msg;
      } catch (const ArgError& e) {
        status = FSIMB_ERR_ARG;
        msg = e.msg;
      } catch (const CudaError& e) {
        status = FSIMB_ERR_CUDA;
        msg = e.msg;
      } catch (const std::bad_alloc&) {
        status = FSIMB_ERR_NOMEM;
        msg = "host allocation failed";
      } catch (const std::exception& e) {
        status = FSIMB_ERR_ARG;
        msg = e.what();
      }
      {
        std::lock_guard<std::mutex> g(mu);
        --planning;
        r->t_planned = Clock::now();
        if (status != FSIMB_OK) {
          r->status = status;
          r->error = msg;
          r->done = true;
          r->t_done = r->t_planned;
          ++stat_failed;
        } else {
          ready.emplace(r->ticket, r);
        }
      }
      work_cv.notify_all();
      if (status != FSIMB_OK) done_cv.notify_all();
    }
  }

  static void CUDART_CB on_wave_done(void* p) {
    Slot* s = static_cast<Slot*>(p);
    s->finished.store(true);
    s->owner->work_cv.notify_all();
  }

  // Lays out and launches the wave of slot s (mu not held).
  void launch(Slot& s) {
    // classes: one per sweep shape among the wave's circuits
    std::vector<ClassShape> shapes;
    s.jobs.clear();
    for (Request* r : s.wave) {
      ResidentCircuit& c = circuit(r->circuit);
      int cls = -1;
      for (size_t k = 0; k < shapes.size(); ++k)
        if (shapes[k].M == c.shape.M && shapes[k].threads == c.shape.threads && shapes[k].occ == c.shape.occ)
          cls = (int)k;
      if (cls < 0) {
        cls = (int)shapes.size();
        shapes.push_back(c.shape);
      }
      r->job.cls = cls;
      s.jobs.push_back(r->job);
    }
    std::lock_guard<std::mutex> g(attr_mu);
    s.exec.layout(s.jobs, shapes, false, s.stream);
    s.exec.apply_attributes();
    CK(cudaEventRecord(s.e0, s.stream));
    s.exec.enqueue(s.stream, false, false, nullptr);
    s.exec.fetch_async(s.stream);
    CK(cudaEventRecord(s.e1, s.stream));
    CK(cudaLaunchHostFunc(s.stream, on_wave_done, &s));
  }

  // Takes the results of slot s's finished wave (mu held).
  void finish(Slot& s) {
    const auto now = Clock::now();
    int kerr = s.exec.read_err();
    float gpu = 0;
    cudaEventElapsedTime(&gpu, s.e0, s.e1);
    stat_busy_ms += gpu;
    double work = 0;
    for (Request* r : s.wave) work += r->work;
    if (gpu > 1.0f && work > 0) gwe_per_ms = 0.8 * gwe_per_ms + 0.2 * (work / gpu);
    for (size_t i = 0; i < s.wave.size(); ++i) {
      Request* r = s.wave[i];
      if (kerr) {
        r->status = FSIMB_ERR_CUDA;
        r->error = "a sweep kernel reached its wait limit for a record copy; results discarded";
        ++stat_failed;
      } else {
        r->results.resize(r->job.F);
        s.exec.results(i, s.jobs[i], r->results.data());
        ++stat_completed;
        stat_fault_patterns += (double)r->job.F * (double)r->pats.P;
        lat_ms.push_back(ms_between(r->t_submit, now));
        queue_ms.push_back(ms_between(r->t_submit, r->t_launch));
        gpu_ms.push_back(gpu);
      }
      r->t_done = now;
      r->done = true;
      // the plan is no longer needed
      r->plan = Plan();
    }
    stat_last_done = now;
    s.wave.clear();
    s.busy = false;
  }

  void dispatch_loop() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> g(mu);
    for (;;) {
      bool progressed = false;
      for (auto& sp : slots) {
        Slot& s = *sp;
        if (s.busy && s.finished.load()) {
          finish(s);
          progressed = true;
          done_cv.notify_all();
        }
      }
      for (auto& sp : slots) {
        Slot& s = *sp;
        if (s.busy || ready.empty()) continue;
        WaveBytes need = overhead();
        const uint32_t max_n = opts.max_wave_requests ? opts.max_wave_requests : 256;
        // The oldest ready request leads the wave (a single admitted request
        // always fits an empty slot).  Later ones join in ticket order while
        // the wave fits the slot and its predicted time stays within
        // max_wave_ms, so small requests are not held up behind a large one
        // in the same wave; one that does not fit lets later, smaller ones
        // try (at most 128 looked at).
        const double max_ms = opts.max_wave_ms ? (double)opts.max_wave_ms : 200.0;
        double wave_ms = 0;
        size_t looked = 0;
        for (auto it = ready.begin(); it != ready.end() && s.wave.size() < max_n && looked < 128;
             ++looked) {
          WaveBytes next = need;
          add(next, it->second->bytes);
          const double ms = it->second->work / gwe_per_ms;
          if (!fits(next, s.cap) || (!s.wave.empty() && wave_ms + ms > max_ms)) {
            ++it;
            continue;
          }
          need = next;
          wave_ms += ms;
          s.wave.push_back(it->second);
          it = ready.erase(it);
        }
        if (s.wave.empty()) continue;
        const auto now = Clock::now();
        for (Request* r : s.wave) r->t_launch = now;
        s.busy = true;
        s.finished.store(false);
        ++stat_waves;
        stat_wave_requests += s.wave.size();
        g.unlock();
        int status = FSIMB_OK;
        std::string msg;
        try {
          launch(s);
        } catch (const CudaError& e) {
          status = FSIMB_ERR_CUDA;
          msg = e.msg;
        } catch (const LimitError& e) {
          status = FSIMB_ERR_LIMIT;
          msg = e.msg;
        } catch (const std::exception& e) {
          status = FSIMB_ERR_ARG;
          msg = e.what();
        }
        g.lock();
        if (status != FSIMB_OK) {
          cudaStreamSynchronize(s.stream);
          for (Request* r : s.wave) {
            r->status = status;
            r->error = msg;
            r->done = true;
            r->t_done = Clock::now();
            ++stat_failed;
          }
          s.wave.clear();
          s.busy = false;
          done_cv.notify_all();
        }
        progressed = true;
      }
      bool busy = false;
      for (auto& sp : slots) busy |= sp->busy;
      if (stopping && !busy && ready.empty() && to_plan.empty() && planning == 0) return;
      if (!progressed) work_cv.wait_for(g, std::chrono::microseconds(500));
    }
  }

  int wait(uint64_t ticket, fsimb_fault_result* out, uint64_t n, int64_t timeout_ms) {
    std::unique_lock<std::mutex> g(mu);
    auto it = requests.find(ticket);
    if (it == requests.end()) throw ArgError{"unknown ticket " + std::to_string(ticket)};
    Request* r = it->second.get();
    auto pred = [&] { return r->done; };
    if (timeout_ms < 0)
      done_cv.wait(g, pred);
    else if (!done_cv.wait_for(g, std::chrono::milliseconds(timeout_ms), pred))
      return FSIMB_ERR_TIMEOUT;
    if (r->status != FSIMB_OK) {
      const int st = r->status;
      err = r->error;
      requests.erase(it);
      return st;
    }
    if (out) {
      if (n < r->results.size()) throw ArgError{"result buffer holds " + std::to_string(n) + " of " +
                                                std::to_string(r->results.size()) + " faults"};
      std::copy(r->results.begin(), r->results.end(), out);
    }
    requests.erase(it);
    return FSIMB_OK;
  }
};

namespace fsimb {

void BatchExec::fetch_async(cudaStream_t s) {
  const uint64_t Fp = std::max<uint64_t>(F_total, 1);
  char* hb = h_res.as<char>();
  if (F_total) {
    CK(cudaMemcpyAsync(hb, d_count, F_total * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hb + Fp * 8, d_first, F_total * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hb + Fp * 16, d_lastflag, F_total, cudaMemcpyDeviceToHost, s));
  }
  CK(cudaMemcpyAsync(hb + Fp * 17, d_ctl.p, sizeof(int), cudaMemcpyDeviceToHost, s));
}

int BatchExec::read_err() const {
  const uint64_t Fp = std::max<uint64_t>(F_total, 1);
  int kerr = 0;
  std::memcpy(&kerr, h_res.as<char>() + Fp * 17, sizeof(int));
  return kerr;
}

}  // namespace fsimb

// -------------------------------------------------------------------- C ABI
extern "C" {

static thread_local std::string g_server_create_error;

int fsimb_server_create(int device, const fsimb_server_opts* opts, fsimb_server** out) {
  if (!out) return FSIMB_ERR_ARG;
  *out = nullptr;
  fsimb_server* s = nullptr;
  try {
    fsimb_server_opts o{};
    if (opts) {
      if (opts->struct_size != 0 && opts->struct_size < sizeof(fsimb_server_opts)) {
        g_server_create_error = "fsimb_server_opts.struct_size too small";
        return FSIMB_ERR_ARG;
      }
      o = *opts;
    }
    if (o.slots > 8) {
      g_server_create_error = "slots must be 0..8";
      return FSIMB_ERR_ARG;
    }
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || device < 0 || device >= n) {
      cudaGetLastError();
      g_server_create_error = std::string("no usable CUDA device ") + std::to_string(device);
      return FSIMB_ERR_CUDA;
    }
    s = new fsimb_server();
    s->device = device;
    s->opts = o;
    CK(cudaSetDevice(device));
    int v = 0;
    CK(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
    s->n_sms = v;
    CK(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    s->smem_optin = (size_t)v;
    CK(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device));
    s->smem_per_sm = (size_t)v;
    s->start();
    *out = s;
    return FSIMB_OK;
  } catch (const CudaError& e) {
    g_server_create_error = e.msg;
    delete s;
    return FSIMB_ERR_CUDA;
  } catch (const std::bad_alloc&) {
    g_server_create_error = "host allocation failed";
    delete s;
    return FSIMB_ERR_NOMEM;
  }
}

int fsimb_server_destroy(fsimb_server* s) {
  delete s;
  return FSIMB_OK;
}

const char* fsimb_server_last_error(const fsimb_server* s) {
  return s ? s->err.c_str() : g_server_create_error.c_str();
}

int fsimb_server_add_circuit(fsimb_server* s, const char* ckt, size_t ckt_len, const uint64_t* words,
                             uint64_t n_patterns, uint32_t* id) {
  API_BEGIN(s)
  if (!ckt || !id) throw ArgError{"null argument"};
  CK(cudaSetDevice(s->device));
  *id = s->add_circuit(ckt, ckt_len, words, n_patterns);
  API_END(s)
}

int fsimb_server_submit(fsimb_server* s, const fsimb_request* req, uint64_t* ticket) {
  API_BEGIN(s)
  if (!req || !ticket) throw ArgError{"null argument"};
  if (req->struct_size != 0 && req->struct_size < sizeof(fsimb_request))
    throw ArgError{"fsimb_request.struct_size too small"};
  *ticket = s->submit(*req);
  API_END(s)
}

int fsimb_server_wait(fsimb_server* s, uint64_t ticket, fsimb_fault_result* out, uint64_t n,
                      int64_t timeout_ms) {
  if (!s) return FSIMB_ERR_ARG;
  try {
    return s->wait(ticket, out, n, timeout_ms);
  } catch (const ArgError& e) {
    s->err = e.msg;
    return FSIMB_ERR_ARG;
  }
}

int fsimb_server_get_stats(fsimb_server* s, fsimb_server_stats* out) {
  if (!s || !out) return FSIMB_ERR_ARG;
  std::lock_guard<std::mutex> g(s->mu);
  *out = fsimb_server_stats{};
  out->completed = s->stat_completed;
  out->failed = s->stat_failed;
  out->waves = s->stat_waves;
  out->mean_wave_requests = s->stat_waves ? (double)s->stat_wave_requests / s->stat_waves : 0.0;
  out->fault_patterns = s->stat_fault_patterns;
  out->ms_gpu_busy = s->stat_busy_ms;
  if (s->stat_any && s->stat_completed)
    out->wall_ms = ms_between(s->stat_first_submit, s->stat_last_done);
  auto q = [](std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const size_t k = std::min(v.size() - 1, (size_t)(p * (double)(v.size() - 1) + 0.5));
    return v[k];
  };
  out->latency_p50_ms = q(s->lat_ms, 0.50);
  out->latency_p99_ms = q(s->lat_ms, 0.99);
  out->latency_max_ms = q(s->lat_ms, 1.0);
  double sum = 0;
  for (double x : s->lat_ms) sum += x;
  out->latency_mean_ms = s->lat_ms.empty() ? 0.0 : sum / s->lat_ms.size();
  out->queue_p50_ms = q(s->queue_ms, 0.50);
  out->queue_p99_ms = q(s->queue_ms, 0.99);
  out->wave_gpu_p50_ms = q(s->gpu_ms, 0.50);
  out->wave_gpu_p99_ms = q(s->gpu_ms, 0.99);
  uint64_t dev = 0;
  {
    std::lock_guard<std::mutex> gc(s->circuits_mu);
    out->circuits = s->circuits.size();
    for (auto& c : s->circuits) dev += c->device_bytes();
  }
  out->resident_bytes = dev;
  for (auto& sl : s->slots) out->slot_bytes += sl->exec.device_bytes();
  return FSIMB_OK;
}

int fsimb_server_reset_stats(fsimb_server* s) {
  if (!s) return FSIMB_ERR_ARG;
  std::lock_guard<std::mutex> g(s->mu);
  s->lat_ms.clear();
  s->queue_ms.clear();
  s->gpu_ms.clear();
  s->stat_completed = s->stat_failed = s->stat_waves = s->stat_wave_requests = 0;
  s->stat_fault_patterns = 0;
  s->stat_busy_ms = 0;
  s->stat_any = false;
  return FSIMB_OK;
}

}  // extern "C"
