/*
 * CPU oracle for the stuck-at fault-simulation path -- TEST INFRASTRUCTURE.
 *
 * This is a plain-C restatement of LSIM's CPU simulator (fsim/simulation.cpp).
 * It is the checker that the GPU path is compared against: only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark may load it, and
 * never as the thing that is measured or shipped.
 *
 * Pinning: the restatement is checked against the golden vectors of the
 * reference's own unit tests (unittests/test_basics.cpp:8-345) and against the
 * reference simulator itself, compiled from its sources by oracle/Makefile
 * into oracle/_ref/ (tests/test_oracle_ref.py).
 *
 * Per-fault results, derived from the reference's per-round PO words
 * (fsim/simulation.cpp:104-147):
 *   detected  - some pattern distinguishes the faulty machine at a PO;
 *   first     - lowest detecting pattern index (-1 if none); bit b of round rd
 *               with `bits` valid bits is pattern rd*64 + bits-1-b (the
 *               MSB-first packing of fsim/generate_fault_patterns.py:66-78);
 *   count     - number of detecting patterns;
 *   ref_flag / ref_rd - the reference's own found_fault_to_pattern entry,
 *               which keeps only the last round (fsim/simulation.cpp:141-144).
 */
#ifndef FSIM_ORACLE_H
#define FSIM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_netlist or_netlist;

typedef struct {
  uint8_t detected;
  uint8_t ref_flag;
  uint8_t pad[6];
  int64_t first;
  uint64_t count;
  uint64_t ref_rd;
} or_result;

typedef struct {
  uint64_t site; /* topological index */
  uint32_t pin;  /* 0 = output, k = k-th input (1-based) */
  uint32_t value;
} or_fault;

/* Parse .ckt text; returns NULL and fills err on failure. */
or_netlist* or_parse_ckt(const char* text, size_t len, char* err, size_t errlen);
void or_free(or_netlist* nl);

uint64_t or_num_elements(const or_netlist* nl);
uint64_t or_num_pis(const or_netlist* nl);
uint64_t or_num_pos(const or_netlist* nl);
uint64_t or_num_gates(const or_netlist* nl);
uint64_t or_num_levels(const or_netlist* nl);
/* Copies of the reference accessors (fsim/simulation.hpp:69-94). */
void or_tpg(const or_netlist* nl, uint64_t* out);            /* [N] */
void or_levels(const or_netlist* nl, uint64_t* out);         /* [N] */
void or_per_level(const or_netlist* nl, uint64_t* out);      /* [n_levels] */
void or_types(const or_netlist* nl, uint8_t* out);           /* [N] */

/* Parse .flst text (plain, or "@pins" extended form) into topological faults. */
int64_t or_parse_flst(const or_netlist* nl, const char* text, size_t len, or_fault* out,
                      size_t cap, char* err, size_t errlen);
/* Parse .ptn text into words [W][nPI]; returns P or -1. */
int64_t or_parse_ptn(const or_netlist* nl, const char* text, size_t len, uint64_t* out,
                     size_t cap, char* err, size_t errlen);

/* Good-machine values of all elements for one round, masked to the round's
 * valid bits (fsim/simulation.cpp:149-184). */
void or_good_values(const or_netlist* nl, const uint64_t* words, uint64_t P, uint64_t rd,
                    uint64_t* out);

/* Fault simulation over rounds [rd0, rd1) for faults [f0, f1).  mode 0 is the
 * reference's full re-simulation per fault (fsim/simulation.cpp:186-228); mode
 * 1 propagates only through the fault's fanout cone (same results); mode 2 is
 * mode 1 over chunks of rounds at once (same results, for large circuits).
 * n_threads > 1 shards faults across POSIX threads.  Results are accumulated
 * into res[f - f0] (initialise with or_results_init). */
void or_results_init(or_result* res, size_t n);
void or_simulate(const or_netlist* nl, const or_fault* faults, uint64_t f0, uint64_t f1,
                 const uint64_t* words, uint64_t P, uint64_t rd0, uint64_t rd1, int mode,
                 int n_threads, or_result* res);

#ifdef __cplusplus
}
#endif

#endif
