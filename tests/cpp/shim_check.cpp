// Exercises include/fsimb.hpp like a caller of fsim::Simulator would:
//   shim_check <device> <ckt> <flst> <ptn> <dot_out>
// Prints the accessors' values one line each ("name v0 v1 ..."); device -1
// skips run().  A read() failure prints "error: <what>" and exits 2.
#include <cstdio>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "fsimb.hpp"

static void put(const char* name, const std::vector<size_t>& v) {
  std::cout << name;
  for (size_t x : v) std::cout << ' ' << x;
  std::cout << '\n';
}

int main(int argc, char** argv) {
  if (argc < 6) {
    std::cerr << "usage: shim_check <device> <ckt> <flst> <ptn> <dot_out>\n";
    return 1;
  }
  const int device = std::stoi(argv[1]);
  fsimb::Simulator sim(device);
  try {
    sim.read(argv[2], argv[3], argv[4]);
  } catch (const std::runtime_error& e) {
    std::cout << "error: " << e.what() << '\n';
    return 2;
  }
  std::cout << "num " << sim.num_PIs() << ' ' << sim.num_POs() << ' ' << sim.num_gates() << ' '
            << sim.num_wires() << ' ' << sim.num_rounds() << '\n';
  put("tpg", sim.gate_idx_to_tpg_order_idx());
  put("per_level", sim.num_gates_per_level());
  {
    std::vector<size_t> idx, lvl, typ;
    for (size_t i = 0; i < sim.num_PIs(); ++i) {
      idx.push_back(sim.pi(i).idx());
      lvl.push_back(sim.pi(i).level());
      typ.push_back((size_t)sim.pi(i).type());
    }
    for (const auto& g : sim.gates()) {
      idx.push_back(g.idx());
      lvl.push_back(g.level());
      typ.push_back((size_t)g.type());
    }
    for (size_t i = 0; i < sim.num_POs(); ++i) {
      idx.push_back(sim.po(i).idx());
      lvl.push_back(sim.po(i).level());
      typ.push_back((size_t)sim.po(i).type());
    }
    put("elem_idx", idx);
    put("elem_level", lvl);
    put("elem_type", typ);
    const bool names = sim.gateTypeToString(fsimb::GateType::NAND) == "NAND" &&
                       sim.gateTypeToString(fsimb::GateType::PO) == "PO" &&
                       sim.gateTypeToString((fsimb::GateType)42) == "UNKNOWN";
    std::cout << "type_names_ok " << (names ? 1 : 0) << '\n';
  }
  sim.visualization_graph(argv[5]);
  if (device >= 0) {
    sim.run(fsimb::Simulator::Mode::SEQUENTIAL, 1);
    put("g_pi", sim.g_pi_results());
    put("g_gate", sim.g_gate_results());
    put("g_po", sim.g_po_results());
    std::vector<size_t> ov;
    for (const auto& g : sim.gates()) ov.push_back(g.output_value());
    put("gate_output_values", ov);
    put("found", sim.found_fault_to_pattern());
    std::vector<size_t> first;
    for (const auto& r : sim.results()) first.push_back((size_t)(r.first_pattern + 1));
    put("first_plus_1", first);
  }
  return 0;
}
