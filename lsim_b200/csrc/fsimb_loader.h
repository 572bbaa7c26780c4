// Fast .ckt loader (fsimb_loader.cu): parallel tokenizing on the host,
// pin-slot table, element order, levels and CSRs on the device.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "fsimb_netlist.h"

namespace fsimb {

struct LoadInfo {
  bool on_device = false;   // the netlist was built by parse_ckt_device
  bool handed_back = false;  // parse_ckt_device declined and the host reader ran
  int threads = 0;          // tokenizer threads
  uint32_t waves = 0;       // element-order waves (longest path from the PIs + 1)
  double ms_total = 0, ms_tokenize = 0, ms_device = 0;
};

// Builds the Netlist parse_ckt builds for the same text, on `device` and
// stream `s`.  Returns false, leaving `nl` untouched, for every text the
// host reader rejects and for netlists whose levels are not sorted in
// element order: the caller then runs parse_ckt, which reports the error or
// builds the schedule levels.
bool parse_ckt_device(const char* text, size_t len, Netlist& nl, int device, cudaStream_t s, int threads,
                      LoadInfo& info);

// Texts at least this long are loaded by parse_ckt_device in the automatic
// mode (a device handle).
constexpr size_t kDeviceLoadBytes = 4u << 20;

}  // namespace fsimb
