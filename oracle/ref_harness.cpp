// Tier-1 oracle harness -- TEST INFRASTRUCTURE.
//
// Drives LSIM's own, unmodified CPU simulator (fsim/simulation.cpp, compiled
// from the reference sources by oracle/Makefile; nothing of it is copied here)
// through the friend hook the reference declares for partitioners
// (fsim/simulation.hpp:41, fsim/pattern.hpp:19, fsim/fault.hpp:19).
//
//   ref_load_text   - Simulator::read(istream, istream, istream), the public
//                     reader (fsim/simulation.cpp:37-63);
//   ref_load_words  - the reader's _read_graph/_read_fault with the pattern
//                     rows stored in file order, which avoids the row
//                     placement of fsim/simulation.cpp:968-969 when
//                     ceil(P/64) > nPI;
//   ref_run_table   - Simulator::run(mode, threads), the public entry point,
//                     returning found_fault_to_pattern and the good values;
//   ref_simulate    - per round _run_good_case, per fault _run_bad_case, and
//                     the masked PO words folded into per-fault detected /
//                     first / count (the reference computes them but keeps
//                     only the last round, fsim/simulation.cpp:131-145).
//                     Faults are sharded over threads, one Simulator each.
#include <barrier>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "fsim/simulation.hpp"

// Friend of Pattern / Fault / ElementBase (declared at global scope there).
class CPUPartitioner {
 public:
  static std::vector<size_t>& words(Pattern& p) { return p._value; }
  static size_t site(const Fault<size_t>& f) { return f._gate_with_fault; }
  static size_t value(const Fault<size_t>& f) { return f._gate_SA_fault_val; }
};

struct ref_result {
  uint8_t detected;
  uint8_t ref_flag;
  uint8_t pad[6];
  int64_t first;
  uint64_t count;
  uint64_t ref_rd;
};

namespace fsim {

// Friend of fsim::Simulator.
class CPUPartitioner {
 public:
  static void load_words(Simulator& s, const std::string& ckt, const std::string& flst,
                         const uint64_t* words, uint64_t P) {
    std::istringstream ick(ckt), ifl(flst);
    ick >> s._num_PIs >> s._num_POs >> s._num_inner_gates >> s._num_wires;
    s._read_graph(ick);
    ifl >> s._num_fault;
    s._read_fault(ifl);
    s._num_pattern = P;
    s._num_rounds = (P + SIZE_T_BITS - 1) / SIZE_T_BITS;
    s._patterns.assign(s._num_rounds, Pattern());
    for (size_t r = 0; r < s._num_rounds; ++r) {
      auto& v = ::CPUPartitioner::words(s._patterns[r]);
      v.assign(words + r * s._num_PIs, words + (r + 1) * s._num_PIs);
    }
  }

  static void simulate(Simulator& s, size_t f0, size_t f1, size_t rd0, size_t rd1,
                       ref_result* res) {
    s._g_pi_results.resize(s._num_PIs);
    s._g_gate_results.resize(s._num_inner_gates);
    s._g_po_results.resize(s._num_POs);
    s._b_pi_results.resize(s._num_PIs);
    s._b_gate_results.resize(s._num_inner_gates);
    s._b_po_results.resize(s._num_POs);
    const size_t last = s._num_rounds ? s._num_rounds - 1 : 0;
    for (size_t rd = rd0; rd < rd1; ++rd) {
      // same formula as fsim/simulation.cpp:115-118
      size_t bits = ((s._num_pattern / (SIZE_T_BITS * (rd + 1)))) ? SIZE_T_BITS
                                                                   : (s._num_pattern % SIZE_T_BITS);
      s._run_good_case(s._patterns[rd], bits);
      for (size_t f = f0; f < f1; ++f) {
        s._run_bad_case(s._faults[f], s._patterns[rd], bits);
        uint64_t diff = 0;
        for (size_t i = 0; i < s._num_POs; ++i) diff |= s._g_po_results[i] ^ s._b_po_results[i];
        ref_result& r = res[f - f0];
        if (diff) {
          r.detected = 1;
          r.count += (uint64_t)__builtin_popcountll(diff);
          int64_t b = 63 - __builtin_clzll(diff);
          int64_t idx = (int64_t)(rd * 64 + bits - 1) - b;
          if (r.first < 0 || idx < r.first) r.first = idx;
        }
        if (rd == last) {
          r.ref_flag = diff != 0;
          r.ref_rd = rd;
        }
      }
    }
  }

  static size_t num_faults(const Simulator& s) { return s._faults.size(); }
  static const std::vector<Fault<size_t>>& faults(const Simulator& s) { return s._faults; }
};

}  // namespace fsim

struct ref_handle {
  std::string ckt, flst;
  std::vector<uint64_t> words;
  uint64_t P = 0;
  bool text_mode = false;
  std::string ptn;
  fsim::Simulator sim;
  std::string err;
  // one Simulator per worker thread, loaded once and reused
  std::vector<std::unique_ptr<fsim::Simulator>> pool;
  double last_seconds = 0;
};

extern "C" {

void* ref_load_text(const char* ckt, size_t ckt_len, const char* flst, size_t flst_len,
                    const char* ptn, size_t ptn_len) {
  ref_handle* h = new ref_handle();
  h->ckt.assign(ckt, ckt_len);
  h->flst.assign(flst, flst_len);
  h->ptn.assign(ptn, ptn_len);
  h->text_mode = true;
  std::istringstream a(h->ckt), b(h->flst), c(h->ptn);
  h->sim.read(a, b, c);
  h->P = 0;
  return h;
}

void* ref_load_words(const char* ckt, size_t ckt_len, const char* flst, size_t flst_len,
                     const uint64_t* words, uint64_t P, uint64_t n_pi) {
  ref_handle* h = new ref_handle();
  h->ckt.assign(ckt, ckt_len);
  h->flst.assign(flst, flst_len);
  h->words.assign(words, words + ((P + 63) / 64) * n_pi);
  h->P = P;
  fsim::CPUPartitioner::load_words(h->sim, h->ckt, h->flst, h->words.data(), P);
  return h;
}

void ref_free(void* hp) { delete (ref_handle*)hp; }

uint64_t ref_num(void* hp, int what) {
  auto& s = ((ref_handle*)hp)->sim;
  switch (what) {
    case 0: return s.num_PIs();
    case 1: return s.num_POs();
    case 2: return s.num_gates();
    case 3: return s.num_wires();
    case 4: return s.num_rounds();
    case 5: return fsim::CPUPartitioner::num_faults(s);
    case 6: return s.num_gates_per_level().size();
  }
  return 0;
}

// tpg [N], levels [N], per-level [L], fault sites/values [2F], pattern words [R*nPI]
void ref_arrays(void* hp, uint64_t* tpg, uint64_t* levels, uint64_t* per_level,
                uint64_t* faults, uint64_t* pwords) {
  auto& s = ((ref_handle*)hp)->sim;
  const auto& t = s.gate_idx_to_tpg_order_idx();
  if (tpg) std::copy(t.begin(), t.end(), tpg);
  if (levels) {
    size_t k = 0;
    for (size_t i = 0; i < s.num_PIs(); ++i) levels[k++] = s.pi(i).level();
    for (size_t i = 0; i < s.num_gates(); ++i) levels[k++] = s.gate(i).level();
    for (size_t i = 0; i < s.num_POs(); ++i) levels[k++] = s.po(i).level();
  }
  if (per_level) {
    const auto& p = s.num_gates_per_level();
    std::copy(p.begin(), p.end(), per_level);
  }
  if (faults) {
    const auto& f = fsim::CPUPartitioner::faults(s);
    for (size_t i = 0; i < f.size(); ++i) {
      faults[2 * i] = ::CPUPartitioner::site(f[i]);
      faults[2 * i + 1] = ::CPUPartitioner::value(f[i]);
    }
  }
  if (pwords) {
    const auto& ps = s.patterns();
    size_t k = 0;
    for (auto& p : ps)
      for (size_t v : p.output_value()) pwords[k++] = v;
  }
}

// Public entry point: Simulator::visualization_graph(path).
void ref_visualize(void* hp, const char* path) {
  ((ref_handle*)hp)->sim.visualization_graph(path);
}

// Public entry point: Simulator::run(mode, threads).
void ref_run_table(void* hp, int mode, int threads, uint64_t* table, uint64_t* good) {
  auto& s = ((ref_handle*)hp)->sim;
  s.run(static_cast<fsim::Simulator::Mode>(mode), (size_t)threads);
  const auto& t = s.found_fault_to_pattern();
  std::copy(t.begin(), t.end(), table);
  if (good) {
    size_t k = 0;
    for (size_t v : s.g_pi_results()) good[k++] = v;
    for (size_t v : s.g_gate_results()) good[k++] = v;
    for (size_t v : s.g_po_results()) good[k++] = v;
  }
}

// Per-fault results over faults [f0,f1) and rounds [rd0,rd1), sharded over
// n_threads Simulators.  The worker Simulators are loaded once (in parallel)
// and kept; ref_seconds() returns the simulation time of the last call,
// measured from the moment every worker is ready to the last one finishing.
void ref_simulate(void* hp, uint64_t f0, uint64_t f1, uint64_t rd0, uint64_t rd1,
                  int n_threads, ref_result* out) {
  ref_handle* h = (ref_handle*)hp;
  for (uint64_t f = f0; f < f1; ++f) {
    std::memset(&out[f - f0], 0, sizeof(ref_result));
    out[f - f0].first = -1;
  }
  if (n_threads <= 1 || f1 - f0 < 2) {
    auto t0 = std::chrono::steady_clock::now();
    fsim::CPUPartitioner::simulate(h->sim, f0, f1, rd0, rd1, out);
    h->last_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return;
  }
  if ((uint64_t)n_threads > f1 - f0) n_threads = (int)(f1 - f0);
  while ((int)h->pool.size() < n_threads) h->pool.emplace_back(nullptr);
  std::vector<std::thread> th;
  std::barrier sync(n_threads + 1);
  uint64_t per = (f1 - f0 + n_threads - 1) / n_threads;
  for (int t = 0; t < n_threads; ++t) {
    uint64_t a = std::min<uint64_t>(f1, f0 + t * per), b = std::min<uint64_t>(f1, a + per);
    th.emplace_back([h, t, a, b, rd0, rd1, f0, out, &sync]() {
      auto& s = h->pool[t];
      if (!s) {
        s.reset(new fsim::Simulator());
        if (h->text_mode) {
          std::istringstream x(h->ckt), y(h->flst), z(h->ptn);
          s->read(x, y, z);
        } else {
          fsim::CPUPartitioner::load_words(*s, h->ckt, h->flst, h->words.data(), h->P);
        }
      }
      sync.arrive_and_wait();
      if (a < b) fsim::CPUPartitioner::simulate(*s, a, b, rd0, rd1, out + (a - f0));
    });
  }
  sync.arrive_and_wait();
  auto t0 = std::chrono::steady_clock::now();
  for (auto& t : th) t.join();
  h->last_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

double ref_seconds(void* hp) { return ((ref_handle*)hp)->last_seconds; }

}  // extern "C"
