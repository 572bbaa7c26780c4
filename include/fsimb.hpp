/*
 * fsimb.hpp -- header-only C++ mirror of LSIM's fsim::Simulator
 * (fsim/simulation.hpp:39-188) over the C ABI of fsimb.h.
 *
 * A caller of the reference changes `#include "fsim/simulation.hpp"` to
 * `#include "fsimb.hpp"` and `fsim::Simulator` to `fsimb::Simulator`; the
 * method names, argument meanings, return types of the accessors and the
 * exceptions of read() are the reference's:
 *   read(path, path, path)  throws std::runtime_error("cannot open circut
 *                           file <path>") etc. (fsim/simulation.cpp:24-32)
 *   read(istream&, istream&, istream&)
 *   run(Mode, num_threads)  every mode runs on the B200 (Mode::CUDA_B200 is
 *                           the same run; num_threads is accepted and unused)
 *   g_pi/g_gate/g_po_results(), found_fault_to_pattern(),
 *   gate_idx_to_tpg_order_idx(), num_gates_per_level(), num_PIs/... ,
 *   pi(i)/gate(i)/po(i)/gates() with idx()/level()/output_value(),
 *   gateTypeToString(type), visualization_graph(path)
 * Beyond the reference: results() gives per fault the detected flag, first
 * detecting pattern and detection count.  Errors other than a missing file
 * throw fsimb::Error (a std::runtime_error) carrying the status code.
 * Like the reference object, a Simulator is not copyable.
 */
#ifndef FSIMB_HPP
#define FSIMB_HPP

#include <fstream>
#include <istream>
#include <iterator>
#include <stdexcept>
#include <string>
#include <vector>

#include "fsimb.h"

namespace fsimb {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

/* Gate type numbering of fsim/base_ppg.hpp:19-32 (PI and PO follow CLKBUF). */
enum class GateType : int { INV = 0, AND, OR, XOR, NAND, NOR, XNOR, MUX, CLKBUF, PI, PO };

class Simulator {
 public:
  enum class Mode { SEQUENTIAL = 0, PARALLEL_TF, PARALLEL_OMP, CUDA_B200 };

  /* An element as ElementBase's public interface shows it
   * (fsim/base_ppg.hpp:47-50): idx() is the topological index, level() the
   * level; output_value() is the element's good-machine word of the last
   * round after run() and 0 before (the reference leaves there the word of
   * its last faulty-machine simulation). */
  class Element {
   public:
    size_t idx() const { return idx_; }
    size_t level() const { return level_; }
    size_t output_value() const { return value_; }
    GateType type() const { return type_; }

   private:
    friend class Simulator;
    size_t idx_ = 0, level_ = 0, value_ = 0;
    GateType type_ = GateType::INV;
  };

  /* device: CUDA device for run(); -1 for a host-only object that reads and
   * answers the accessors but cannot run. */
  explicit Simulator(int device = 0) {
    if (int rc = fsimb_create(device, &h_)) throw Error(rc, fsimb_last_error(nullptr));
  }
  ~Simulator() { fsimb_destroy(h_); }
  Simulator(const Simulator&) = delete;
  Simulator& operator=(const Simulator&) = delete;

  void read(const std::string& ckt, const std::string& flst, const std::string& ptn) {
    std::ifstream a(ckt), b(flst), c(ptn);
    if (!a) throw std::runtime_error("cannot open circut file " + ckt);
    if (!b) throw std::runtime_error("cannot open fault file " + flst);
    if (!c) throw std::runtime_error("cannot open pattern file " + ptn);
    read(a, b, c);
  }

  void read(std::istream& ckt, std::istream& flst, std::istream& ptn) {
    const std::string a = slurp(ckt), b = slurp(flst), c = slurp(ptn);
    check(fsimb_load_buffers(h_, a.data(), a.size(), b.data(), b.size(), c.data(), c.size()));
    load_introspection();
  }

  void run(Mode mode = Mode::CUDA_B200, size_t num_threads = 1) {
    (void)mode;
    (void)num_threads;
    fsimb_opts o{};
    o.struct_size = sizeof o;
    check(fsimb_run(h_, &o));
    load_results();
  }

  const std::vector<size_t>& g_pi_results() const { return g_pi_; }
  const std::vector<size_t>& g_gate_results() const { return g_gate_; }
  const std::vector<size_t>& g_po_results() const { return g_po_; }
  const std::vector<size_t>& found_fault_to_pattern() const { return found_; }
  const std::vector<fsimb_fault_result>& results() const { return results_; }

  size_t num_PIs() const { return (size_t)info_.num_pis; }
  size_t num_gates() const { return (size_t)info_.num_gates; }
  size_t num_POs() const { return (size_t)info_.num_pos; }
  size_t num_pos() const { return (size_t)info_.num_pos; }
  size_t num_wires() const { return (size_t)info_.num_wires; }
  size_t num_rounds() const { return (size_t)info_.num_rounds; }
  size_t num_faults() const { return (size_t)info_.num_faults; }
  const std::vector<size_t>& gate_idx_to_tpg_order_idx() const { return tpg_; }
  const std::vector<size_t>& num_gates_per_level() const { return per_level_; }

  /* fsim/simulation.hpp:58-63: elements by position among the PIs, gates, POs. */
  Element pi(size_t i) const { return element(i); }
  Element gate(size_t i) const { return element((size_t)info_.num_pis + i); }
  Element po(size_t i) const { return element((size_t)(info_.num_pis + info_.num_gates) + i); }
  std::vector<Element> gates() const {
    std::vector<Element> g;
    for (size_t i = 0; i < (size_t)info_.num_gates; ++i) g.push_back(gate(i));
    return g;
  }
  /* fsim/simulation.cpp:1127-1155 */
  std::string gateTypeToString(GateType type) const {
    static const char* const names[] = {"INV", "AND", "OR",     "XOR", "NAND", "NOR",
                                        "XNOR", "MUX", "CLKBUF", "PI",  "PO"};
    const int t = (int)type;
    return t >= 0 && t <= 10 ? names[t] : "UNKNOWN";
  }

  void visualization_graph(const std::string& output_file) {
    char* text = nullptr;
    size_t len = 0;
    check(fsimb_dot(h_, &text, &len));
    std::ofstream f(output_file);
    f.write(text, (std::streamsize)len);
    fsimb_free_text(text);
  }

  /* Circuit loader for the reads that follow (FSIMB_LOAD_AUTO / _HOST /
   * _DEVICE, tokenizer threads; fsimb_set_loader) and how the last circuit
   * was loaded. */
  void set_loader(int mode, int threads = 0) { check(fsimb_set_loader(h_, mode, threads)); }
  fsimb_load_info load_info() const {
    fsimb_load_info li{};
    check(fsimb_get_load_info(h_, &li));
    return li;
  }

  fsimb_handle* handle() { return h_; }

 private:
  fsimb_handle* h_ = nullptr;
  fsimb_info info_{};
  std::vector<size_t> tpg_, per_level_, levels_, g_pi_, g_gate_, g_po_, found_;
  std::vector<uint8_t> types_;
  std::vector<fsimb_fault_result> results_;

  static std::string slurp(std::istream& s) {
    return std::string(std::istreambuf_iterator<char>(s), std::istreambuf_iterator<char>());
  }

  void check(int rc) const {
    if (rc) throw Error(rc, fsimb_last_error(h_));
  }

  static std::vector<size_t> to_size(const std::vector<uint64_t>& v) {
    return std::vector<size_t>(v.begin(), v.end());
  }

  void load_introspection() {
    check(fsimb_get_info(h_, &info_));
    std::vector<uint64_t> t(info_.num_elements), l(info_.num_levels);
    check(fsimb_topo_map(h_, t.data(), t.size()));
    check(fsimb_gates_per_level(h_, l.data(), l.size()));
    tpg_ = to_size(t);
    per_level_ = to_size(l);
    std::vector<uint64_t> lv(info_.num_elements);
    check(fsimb_levels(h_, lv.data(), lv.size()));
    levels_ = to_size(lv);
    types_.assign(info_.num_elements, 0);
    check(fsimb_types(h_, types_.data(), types_.size()));
    g_pi_.clear();
    g_gate_.clear();
    g_po_.clear();
    found_.clear();
    results_.clear();
  }

  Element element(size_t t) const {
    if (t >= levels_.size()) throw std::out_of_range("element index out of range");
    Element e;
    e.idx_ = t;
    e.level_ = levels_[t];
    e.type_ = (GateType)types_[t];
    const size_t np = g_pi_.size(), ng = g_gate_.size();
    if (t < np)
      e.value_ = g_pi_[t];
    else if (t < np + ng)
      e.value_ = g_gate_[t - np];
    else if (t - np - ng < g_po_.size())
      e.value_ = g_po_[t - np - ng];
    return e;
  }

  void load_results() {
    results_.resize(info_.num_faults);
    check(fsimb_results(h_, results_.data(), results_.size()));
    std::vector<uint64_t> f(2 * info_.num_faults), g(info_.num_elements);
    check(fsimb_found_fault_to_pattern(h_, f.data(), f.size()));
    found_ = to_size(f);
    if (info_.num_rounds) check(fsimb_good_values(h_, info_.num_rounds - 1, g.data(), g.size()));
    const size_t np = (size_t)info_.num_pis, ng = (size_t)info_.num_gates;
    g_pi_.assign(g.begin(), g.begin() + np);
    g_gate_.assign(g.begin() + np, g.begin() + np + ng);
    g_po_.assign(g.begin() + np + ng, g.end());
  }
};

}  // namespace fsimb

#endif  // FSIMB_HPP
