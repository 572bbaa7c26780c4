// Internal declarations shared by the library's translation units: error
// types thrown inside the library and turned into status codes at the C ABI,
// device buffers, and the per-circuit handle (struct fsimb_handle of
// include/fsimb.h).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <functional>
#include <new>
#include <string>
#include <vector>

#include "../../include/fsimb.h"
#include "fsimb_loader.h"
#include "fsimb_netlist.h"
#include "fsimb_plan.h"

namespace fsimb {

struct CudaError {
  std::string msg;
};
struct LimitError {
  std::string msg;
};
struct StateError {
  std::string msg;
};
struct ArgError {
  std::string msg;
};
struct IoError {
  std::string msg;
};

#define CK(call)                                                                            \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::fsimb::CudaError{std::string(#call) + ": " + cudaGetErrorString(e_)};         \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  void ensure(size_t bytes) {
    if (bytes <= n && p) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      throw CudaError{"cudaMalloc(" + std::to_string(bytes) + " bytes): " + cudaGetErrorString(e)};
    }
    n = bytes;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  template <class T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

template <class T>
inline void upload(DevBuf& b, const std::vector<T>& v, cudaStream_t s) {
  b.ensure(v.size() * sizeof(T));
  if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

// Largest sweep CTA for M words per item (the kernels' launch bounds).
inline uint32_t sweep_max_threads(int M) { return M >= 8 ? 512 : (M >= 4 ? 768 : 1024); }

// Sweep CTA size: one thread per gate of a level; the multiple of 32 that
// splits the typical (90th percentile) level width into equal rounds, so no
// thread idles long before the per-level barrier.  `widths` holds the gate
// count of each swept level (reordered in place).
inline uint32_t pick_sweep_threads(std::vector<uint32_t>& widths, int M) {
  const uint32_t tmax = sweep_max_threads(M);
  uint32_t w = 64;
  if (!widths.empty()) {
    std::nth_element(widths.begin(), widths.begin() + widths.size() * 9 / 10, widths.end());
    w = std::max<uint32_t>(widths[widths.size() * 9 / 10], 1);
  }
  uint32_t best = 64;
  double best_cost = 1e30;
  for (uint32_t k = 1; k <= 64; ++k) {
    uint32_t t = (w + k - 1) / k;
    t = std::max<uint32_t>(64, (t + 31) / 32 * 32);
    if (t > tmax) continue;
    const double cost = (double)k * t + 8.0 * k;  // issued slots + per-round overhead
    if (cost < best_cost) {
      best_cost = cost;
      best = t;
    }
  }
  return best;
}

// Dynamic shared memory one sweep CTA may take when `occ` CTAs share an SM
// (each CTA also holds the kernel's static __shared__ variables and the
// 1 KB the hardware reserves per CTA).
inline size_t sweep_smem_share(size_t smem_optin, size_t smem_per_sm, int occ) {
  const size_t static_smem = 512, reserved = 1024;
  const size_t budget = smem_optin > static_smem + reserved ? smem_optin - static_smem - reserved : 0;
  if (occ <= 1) return budget;
  const size_t per = smem_per_sm / (size_t)occ;
  return per > static_smem + reserved ? std::min(budget, per - static_smem - reserved) : 0;
}

// Bytes of a sweep CTA's value slots: max_live slots of M words, 16-byte rounded.
inline uint32_t sweep_vals_bytes(uint32_t max_live, int M) {
  return (uint32_t)(((size_t)max_live * M * 8 + 15) / 16 * 16);
}

// Page-locked host staging buffer.
struct PinnedBuf {
  void* p = nullptr;
  size_t n = 0;
  void ensure(size_t bytes) {
    if (bytes <= n && p) return;
    release();
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocHost(&p, bytes);
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      throw CudaError{"cudaMallocHost(" + std::to_string(bytes) + " bytes): " + cudaGetErrorString(e)};
    }
    n = bytes;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
  template <class T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

// Default sweep shape of a circuit: two CTAs per SM at 8 or 4 words per
// item when the value slots leave room for at least 64 staged records (the
// CTA size then lowered until two fit), else the largest words per item
// whose slots fit one CTA per SM, with the width heuristic's CTA size.
// sched_at(M) returns the schedule at M; occupancy(M, threads, smem) the
// sweep kernel's CTAs per SM.
void default_sweep_shape(const Plan& plan, const std::function<const Schedule&(int)>& sched_at,
                         const std::function<int(int, int, size_t)>& occupancy,
                         std::vector<uint32_t> widths, uint32_t widest, size_t smem_optin,
                         size_t smem_per_sm, int& M, int& occ, int& threads);

// A fresh value for fsimb_handle::gen: every change of a handle's circuit,
// faults or patterns gets a number no other state of any handle had.
uint64_t next_generation();

}  // namespace fsimb

struct fsimb_handle {
  int device = -1;
  int n_sms = 0;
  size_t smem_optin = 0, smem_per_sm = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  uint64_t gen = 0;       // changes whenever circuit, faults or patterns change
  uint64_t plan_gen = 0;  // changes whenever circuit or faults change

  fsimb::Netlist nl;
  bool has_ckt = false;
  std::vector<fsimb::Fault> faults;
  bool has_faults = false;
  fsimb::Patterns pats;
  bool has_pats = false;

  fsimb::Plan plan;
  bool plan_valid = false;
  bool plan_uploaded = false;
  fsimb::Schedule sched;          // for sched_M words per item
  int sched_M = 0;
  bool sched_uploaded = false;
  // Schedules built so far for this plan, per words per item (1, 2, 4, 8).
  fsimb::Schedule sched_cache[4];
  uint64_t sched_cache_gen[4] = {0, 0, 0, 0};
  // Autotuned sweep shape of plan_gen (fsimb_opts.tune).
  uint64_t tuned_gen = 0;
  int tuned_M = 0, tuned_T = 0, tuned_occ = 0;
  cudaEvent_t tune_ev[2] = {nullptr, nullptr};
  // Recorded after each fsimb_run's uploads, on the run's stream: work on
  // another stream that reads the circuit arrays waits for it.
  cudaEvent_t upload_ev = nullptr;

  fsimb::DevBuf d_type, d_fi_off, d_fi_idx, d_recs, d_level, d_level_off, d_li_off, d_li;
  fsimb::DevBuf d_lvl;     // schedule LevelDesc per level
  fsimb::DevBuf d_eflag;   // wide-circuit sweep: per element, evaluated / drives a PO
  fsimb::DevBuf d_gvals;   // wide-circuit sweep: per-CTA value regions
  fsimb::DevBuf d_roots, d_members, d_traced, d_inj, d_exact;
  fsimb::DevBuf d_pwords, d_good, d_out, d_sens, d_count, d_first, d_lastflag, d_queue, d_err;
  fsimb::DevBuf d_root_list[2], d_sweep_list, d_exact_list[2], d_nout, d_tune_list;
  uint64_t good_tiles = 0;  // tiles held in d_good
  uint64_t good_P = 0;
  bool pats_uploaded = false;  // d_pwords holds the current patterns
  bool eflag_uploaded = false; // d_eflag holds the current plan's element flags

  std::vector<fsimb_fault_result> results;
  bool has_results = false;
  fsimb_stats stats{};
  std::vector<cudaEvent_t> events;

  ~fsimb_handle() {
    if (device >= 0) {
      cudaSetDevice(device);
      for (fsimb::DevBuf* b : {&d_type, &d_fi_off, &d_fi_idx, &d_recs, &d_level, &d_level_off,
                        &d_lvl, &d_eflag, &d_gvals, &d_li_off, &d_li, &d_roots, &d_members, &d_traced, &d_inj, &d_exact,
                        &d_pwords, &d_good, &d_out, &d_sens, &d_count, &d_first, &d_lastflag,
                        &d_queue, &d_err, &d_root_list[0], &d_root_list[1], &d_sweep_list,
                        &d_exact_list[0], &d_exact_list[1], &d_nout, &d_tune_list})
        b->release();
      for (auto e : events) cudaEventDestroy(e);
      for (auto e : tune_ev)
        if (e) cudaEventDestroy(e);
      if (upload_ev) cudaEventDestroy(upload_ev);
      if (stream) cudaStreamDestroy(stream);
    }
  }

  cudaEvent_t ev(size_t i) {
    while (events.size() <= i) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      events.push_back(e);
    }
    return events[i];
  }

  uint64_t device_bytes() const {
    uint64_t s = 0;
    for (const fsimb::DevBuf* b : {&d_type, &d_fi_off, &d_fi_idx, &d_recs, &d_level, &d_level_off,
                            &d_lvl, &d_eflag, &d_gvals, &d_li_off, &d_li, &d_roots, &d_members, &d_traced, &d_inj, &d_exact,
                            &d_pwords, &d_good, &d_out, &d_sens, &d_count, &d_first, &d_lastflag,
                            &d_queue, &d_err, &d_root_list[0], &d_root_list[1], &d_sweep_list,
                            &d_exact_list[0], &d_exact_list[1], &d_nout, &d_tune_list})
      s += b->n;
    return s;
  }

  void invalidate_circuit() {
    has_faults = false;
    has_pats = false;
    plan_valid = false;
    plan_uploaded = false;
    sched_M = 0;
    sched_uploaded = false;
    has_results = false;
    good_tiles = 0;
  }

  // Circuit loader (fsimb_set_loader): 0 automatic, 1 host, 2 device.
  int load_mode = 0;
  int load_threads = 0;
  fsimb::LoadInfo load_info;

  void load_ckt(const char* t, size_t n) {
    fsimb::Netlist tmp;
    const bool dev = device >= 0 && (load_mode == 2 || (load_mode == 0 && n >= fsimb::kDeviceLoadBytes));
    const auto t0 = std::chrono::steady_clock::now();
    fsimb::LoadInfo li;
    bool built = false;
    if (dev) {
      try {
        built = fsimb::parse_ckt_device(t, n, tmp, device, stream, load_threads, li);
      } catch (const fsimb::CudaError&) {
        // no room on the device (or the like): the host reader still can
        cudaStreamSynchronize(stream);
        cudaGetLastError();
        built = false;
      }
    }
    if (!built) {
      fsimb::parse_ckt(t, n, tmp);
      li = fsimb::LoadInfo{};
      li.handed_back = dev;
      li.threads = 1;
      li.ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    load_info = li;
    nl = std::move(tmp);
    has_ckt = true;
    gen = plan_gen = fsimb::next_generation();
    invalidate_circuit();
    faults.clear();
    pats = fsimb::Patterns();
  }
  void load_flst(const char* t, size_t n) {
    if (!has_ckt) throw fsimb::StateError{"load a circuit first"};
    std::vector<fsimb::Fault> tmp;
    fsimb::parse_flst(t, n, nl, tmp);
    faults = std::move(tmp);
    has_faults = true;
    gen = plan_gen = fsimb::next_generation();
    plan_valid = false;
    plan_uploaded = false;
    has_results = false;
  }
  void load_ptn(const char* t, size_t n) {
    if (!has_ckt) throw fsimb::StateError{"load a circuit first"};
    fsimb::Patterns tmp;
    fsimb::parse_ptn(t, n, nl, tmp);
    pats = std::move(tmp);
    has_pats = true;
    gen = fsimb::next_generation();
    has_results = false;
    good_tiles = 0;
    pats_uploaded = false;
  }

  void run(const fsimb_opts* opts);
  // The schedule at M words per item for the current plan (cached per M).
  const fsimb::Schedule& cached_schedule(int M);
  // Makes `sched` the schedule at M (re-uploaded before the next sweep).
  void use_schedule(int M);
  // default_sweep_shape for this circuit and the plain sweep kernel.
  void default_shape(std::vector<uint32_t> widths, uint32_t widest, int& M, int& occ, int& threads);
  // Times candidate shapes on a strided sample of tile 0's sweeps and keeps
  // the fastest in tuned_M / tuned_T / tuned_occ.  Needs the plan and the
  // patterns on the device.
  void tune_shape(cudaStream_t s, const std::vector<uint32_t>& widths, uint32_t widest);
};

// Wraps a C ABI body: exceptions become status codes and (h)->err.
#define API_BEGIN(h)                                    \
  if (!(h)) return FSIMB_ERR_ARG;                       \
  try {
#define API_END(h)                                      \
  }                                                     \
  catch (const fsimb::ParseError& e) {                  \
    (h)->err = e.msg;                                   \
    return FSIMB_ERR_PARSE;                             \
  }                                                     \
  catch (const fsimb::CudaError& e) {                   \
    (h)->err = e.msg;                                   \
    return FSIMB_ERR_CUDA;                              \
  }                                                     \
  catch (const fsimb::LimitError& e) {                  \
    (h)->err = e.msg;                                   \
    return FSIMB_ERR_LIMIT;                             \
  }                                                     \
  catch (const fsimb::StateError& e) {                  \
    (h)->err = e.msg;                                   \
    return FSIMB_ERR_STATE;                             \
  }                                                     \
  catch (const fsimb::ArgError& e) {                    \
    (h)->err = e.msg;                                   \
    return FSIMB_ERR_ARG;                               \
  }                                                     \
  catch (const fsimb::IoError& e) {                     \
    (h)->err = e.msg;                                   \
    return FSIMB_ERR_IO;                                \
  }                                                     \
  catch (const std::bad_alloc&) {                       \
    (h)->err = "host allocation failed";                \
    return FSIMB_ERR_NOMEM;                             \
  }                                                     \
  catch (const std::exception& e) {                     \
    (h)->err = e.what();                                \
    return FSIMB_ERR_ARG;                               \
  }                                                     \
  (h)->err.clear();                                     \
  return FSIMB_OK;
