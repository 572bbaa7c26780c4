// Drop-in for LSIM's main/MA_partition.cu:
// `fsimb_ma_partition <ckt> <flst> <ptn> <hypergraph> <out> <rds>`.
//
// Same arguments as MA_cuda_partition (main/MA_partition.cu:20-37); the
// hypergraph and output paths are accepted and unused there as here.  Reads
// the inputs (CUDAMAPartitioner::read), then runs the simulation <rds> times
// (prepare_gpu_simulation + run, cuda_MA_partition.cu:496-538) and prints the
// time of each run.  Unlike the reference's path, which simulates the good
// machine on 32-bit words of the first round only, every run here covers all
// rounds and all faults with 64-bit words.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <iostream>

#include "fsimb.h"

int main(int argc, char** argv) {
  if (argc < 7) {
    std::cerr << "Usage: " << argv[0]
              << " <ckt_path> <flst_path> <ptn_path> <hypergraph_path> <outputfile_path> <num_simulation_rds>\n";
    return 1;
  }
  const long rds = std::atol(argv[6]);
  fsimb_handle* h = nullptr;
  if (fsimb_create(0, &h)) {
    std::cerr << fsimb_last_error(nullptr) << "\n";
    return 1;
  }
  if (fsimb_load_files(h, argv[1], argv[2], argv[3])) {
    std::cerr << fsimb_last_error(h) << "\n";
    fsimb_destroy(h);
    return 1;
  }
  for (long r = 0; r < rds; ++r) {
    auto t0 = std::chrono::steady_clock::now();
    if (fsimb_run(h, nullptr)) {
      std::cerr << fsimb_last_error(h) << "\n";
      fsimb_destroy(h);
      return 1;
    }
    auto t1 = std::chrono::steady_clock::now();
    fsimb_stats st;
    fsimb_get_stats(h, &st);
    std::printf("run %ld: %.3f ms (device %.3f ms: good %.3f, sweeps %.3f, tracing %.3f)\n", r,
                std::chrono::duration<double>(t1 - t0).count() * 1000, st.ms_total, st.ms_good, st.ms_sweep,
                st.ms_ffr);
  }
  fsimb_destroy(h);
  return 0;
}
