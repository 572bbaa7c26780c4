// Drop-in for LSIM's main/simple.cpp: `fsimb_simple <ckt> <flst> <ptn> <out>`.
//
// Reads the three inputs (fsim::Simulator::read), runs the fault simulation on
// the B200, prints the timings and the last round's good-machine word of every
// element as `arr[i] = v` (main/simple.cpp:104-123).  `<out>` receives the
// per-fault results (file id, stuck value, pin, detected, first pattern,
// count, and the reference's found_fault_to_pattern pair); an `<out>` ending
// in ".dot" receives the Graphviz view instead (main/simple.cpp:64-67).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "fsimb.h"

static double round_to(double v, double p) { return std::round(v / p) * p; }

int main(int argc, char** argv) {
  if (argc < 5) {
    std::cerr << "Usage: " << argv[0] << " <ckt> <flst> <ptn> <out>\n";
    return 1;
  }
  fsimb_handle* h = nullptr;
  if (fsimb_create(0, &h)) {
    std::cerr << fsimb_last_error(nullptr) << "\n";
    return 1;
  }
  auto fail = [&](const char* what) {
    std::cerr << what << ": " << fsimb_last_error(h) << "\n";
    fsimb_destroy(h);
    return 1;
  };
  auto t0 = std::chrono::steady_clock::now();
  if (fsimb_load_files(h, argv[1], argv[2], argv[3])) return fail("read");
  auto t1 = std::chrono::steady_clock::now();
  if (fsimb_run(h, nullptr)) return fail("run");
  auto t2 = std::chrono::steady_clock::now();
  fsimb_info info;
  fsimb_get_info(h, &info);
  std::cout << "Execution Time:\n";
  std::cout << "Read Data: " << round_to(std::chrono::duration<double>(t1 - t0).count() * 1000, 0.001)
            << " ms\n";
  std::cout << "CUDA_B200: " << round_to(std::chrono::duration<double>(t2 - t1).count() * 1000, 0.001)
            << " ms\n";
  const std::string out = argv[4];
  if (out.size() >= 4 && out.compare(out.size() - 4, 4, ".dot") == 0) {
    char* text = nullptr;
    size_t len = 0;
    if (fsimb_dot(h, &text, &len)) return fail("dot");
    std::ofstream(out) << std::string(text, len);
    fsimb_free_text(text);
  } else {
    std::vector<fsimb_fault_result> res(info.num_faults);
    std::vector<uint32_t> site(info.num_faults);
    std::vector<uint8_t> pin(info.num_faults), val(info.num_faults);
    std::vector<uint64_t> tpg(info.num_elements), order(info.num_elements);
    if (fsimb_results(h, res.data(), res.size()) ||
        fsimb_faults(h, site.data(), pin.data(), val.data(), site.size()) ||
        fsimb_topo_map(h, tpg.data(), tpg.size()))
      return fail("results");
    for (uint64_t f = 0; f < tpg.size(); ++f) order[tpg[f]] = f;
    std::ofstream o(out);
    o << "# file_id value pin detected first_pattern count ref_flag ref_round\n";
    for (size_t i = 0; i < res.size(); ++i)
      o << order[site[i]] << ' ' << (int)val[i] << ' ' << (int)pin[i] << ' ' << (int)res[i].detected << ' '
        << res[i].first_pattern << ' ' << res[i].count << ' ' << (int)res[i].ref_last_round_flag << ' '
        << res[i].ref_last_rd << '\n';
  }
  if (info.num_rounds) {
    std::vector<uint64_t> arr(info.num_elements);
    if (fsimb_good_values(h, info.num_rounds - 1, arr.data(), arr.size())) return fail("good values");
    for (size_t i = 0; i < arr.size(); ++i) std::cout << "arr[" << i << "] = " << arr[i] << '\n';
  }
  fsimb_destroy(h);
  return 0;
}
