/*
 * fsimb.h -- C ABI of the B200-native stuck-at fault simulator.
 *
 * The library replaces the simulation layer of LSIM (fsim::Simulator,
 * fsim/simulation.hpp:39-188, and CUDAMAPartitioner,
 * fsim/cuda_MA_partition/cuda_MA_partition.cuh:125-260) behind plain C entry
 * points: opaque handle, plain pointers and sizes, an int status on every
 * call (0 = ok) and a per-handle error message.  No exception and no exit()
 * crosses this boundary.  A handle is used by one thread at a time;
 * different handles are independent.  Device memory belongs to the handle.
 *
 * Inputs are LSIM's .ckt / .flst / .ptn text formats with the reference's
 * semantics (element order, fault mapping, pattern rounds).  Results per
 * fault: detected flag, first detecting pattern (-1 if none), detection
 * count, and the reference's own last-round view of found_fault_to_pattern.
 */
#ifndef FSIMB_H
#define FSIMB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define FSIMB_OK 0
#define FSIMB_ERR_ARG 1     /* bad argument or size */
#define FSIMB_ERR_PARSE 2   /* malformed or unsupported input text */
#define FSIMB_ERR_CUDA 3    /* CUDA runtime error or no usable GPU */
#define FSIMB_ERR_STATE 4   /* call order (e.g. results before run) */
#define FSIMB_ERR_NOMEM 5   /* host or device allocation failed */
#define FSIMB_ERR_IO 6      /* file could not be opened or read */
#define FSIMB_ERR_LIMIT 7   /* circuit exceeds a documented limit */
#define FSIMB_ERR_TIMEOUT 8 /* fsimb_server_wait: the request is not done yet */

typedef struct fsimb_handle fsimb_handle;

/* One fault's result (32 bytes). */
typedef struct {
  uint8_t detected;            /* some pattern detects the fault */
  uint8_t ref_last_round_flag; /* found_fault_to_pattern[2f] of the reference */
  uint8_t pad[6];
  int64_t first_pattern;       /* lowest detecting pattern index, -1 if none */
  uint64_t count;              /* detecting patterns (count mode) */
  uint64_t ref_last_rd;        /* found_fault_to_pattern[2f+1] of the reference */
} fsimb_fault_result;

/* Run options.  Zero-initialise and set struct_size = sizeof(fsimb_opts).
 * A struct_size of the first seven fields (the layout before n_detect) is
 * accepted too: the later fields then read as 0. */
typedef struct {
  uint32_t struct_size;
  uint32_t drop;             /* 0: count mode (every pattern); 1: drop a fault
                                after the 2048-pattern tile in which its count
                                reaches n_detect (first_pattern exact, count
                                covers the patterns up to the end of that tile) */
  uint32_t words_per_item;   /* sweep words per work item: 0 auto, or 1,2,4,8
                                (1 or 2 for the wide-circuit sweep) */
  uint32_t block_threads;    /* sweep CTA size: 0 auto, or a multiple of 32 up to 1024 */
  uint32_t ctas_per_sm;      /* sweep CTAs sharing an SM: 0 auto, or 1..8; sizes the
                                record buffer so that many fit */
  uint32_t tune;             /* 1, with the three above 0: on the first run of a circuit and
                                fault list, time candidate sweep shapes on a strided sample
                                of the first tile's sweeps and keep the fastest */
  void* stream;              /* cudaStream_t to run on; NULL: the handle's stream */
  uint32_t n_detect;         /* with drop = 1: detections after which a fault is dropped
                                (N-detect); 0 or 1: the first detection */
  uint32_t sweep_variant;    /* 0 auto: live values in shared memory when they fit, else
                                in global memory; 1 shared memory (FSIMB_ERR_LIMIT when
                                they do not fit); 2 global memory */
  uint32_t wait_test;        /* test hook, normally 0.  1: one sweep CTA waits on a barrier
                                that no copy completes; the wait gives up after 20 ms and
                                the run fails with FSIMB_ERR_CUDA, results discarded, the
                                handle still usable.  Shared-memory sweep only. */
  uint32_t pad;
} fsimb_opts;

/* Sizes of the loaded problem. */
typedef struct {
  uint64_t num_pis, num_pos, num_gates, num_wires;
  uint64_t num_elements;     /* PIs + gates + POs */
  uint64_t num_levels;       /* entries of num_gates_per_level */
  uint64_t num_faults;
  uint64_t num_patterns;
  uint64_t num_rounds;       /* ceil(patterns / 64) */
} fsimb_info;

/* Counters and timings of the last run. */
typedef struct {
  double ms_total, ms_good, ms_sweep, ms_ffr, ms_h2d, ms_d2h;
  uint64_t n_tiles;          /* 2048-pattern tiles */
  uint64_t n_stem_sweeps;    /* FFR roots whose observability is swept */
  uint64_t n_exact_sweeps;   /* faults simulated by an exact sweep (MUX cones) */
  uint64_t n_traced_faults;
  uint64_t n_roots;
  uint64_t sweep_items;      /* (sweep, subtile) work items executed */
  uint64_t dense_gate_words; /* gate-word evaluations done by the sweeps */
  uint64_t sweep_alg_bytes;  /* their algorithmic bytes: 8*(fanin+1) each */
  uint64_t good_gate_words;  /* gate-word evaluations of the good machine */
  uint64_t max_live;         /* shared-memory slots per sweep */
  uint32_t words_per_item, block_threads, blocks, smem_bytes;
  uint64_t device_bytes;     /* device memory held by the handle */
  uint64_t kernel_launches;  /* kernels launched by the last run */
  double ms_compute;         /* device time from results init to the last tile */
  uint64_t bank_conflict_groups; /* sweep access groups whose slots share a bank position */
  uint64_t bank_access_groups;   /* sweep access groups (fanin loads and stores) per item */
  double ms_tune;            /* shape autotuning inside this run (0 when reused) */
  uint32_t ctas_per_sm;      /* sweep CTAs resident per SM */
  uint32_t sweep_variant;    /* 1: live values in shared memory; 2: in global memory */
  uint64_t hbm_bytes_per_tile; /* compulsory DRAM bytes of one sweep launch: the tile's good
                                  words, the schedule (gate records, live-in lists), the
                                  sweep output rows */
} fsimb_stats;

/* Lifecycle.  fsimb_create fails with FSIMB_ERR_CUDA when `device` is not a
 * usable CUDA device; there is no CPU fallback.  device = -1 creates a
 * host-only handle that can load inputs and answer the introspection calls
 * (format checks without a GPU); fsimb_run on it fails with FSIMB_ERR_CUDA. */
int fsimb_create(int device, fsimb_handle** out);
int fsimb_destroy(fsimb_handle* h);
/* Message of the last failed call on h (h may be NULL for fsimb_create). */
const char* fsimb_last_error(const fsimb_handle* h);

/* Loading.  Replaces Simulator::read(path, path, path) and
 * Simulator::read(istream&, istream&, istream&) (fsim/simulation.cpp:12-63).
 * Pattern rows are taken in file order; the reference stores row r at round
 * tpg[r] (fsim/simulation.cpp:968-969), which is the same whenever
 * ceil(P/64) <= nPI and undefined otherwise. */
int fsimb_load_files(fsimb_handle* h, const char* ckt_path, const char* flst_path,
                     const char* ptn_path);
int fsimb_load_buffers(fsimb_handle* h, const char* ckt, size_t ckt_len, const char* flst,
                       size_t flst_len, const char* ptn, size_t ptn_len);
/* Circuit only (clears faults and patterns). */
int fsimb_load_circuit(fsimb_handle* h, const char* ckt, size_t ckt_len);

/* Circuit loader used by the three calls above.  FSIMB_LOAD_AUTO (the
 * default): on a handle with a device, .ckt texts of 4 MiB and more are
 * levelized on the device, smaller ones by the host reader;
 * FSIMB_LOAD_HOST: always the host reader; FSIMB_LOAD_DEVICE: the device
 * loader whenever the handle has a device.  The device loader tokenizes on
 * `threads` host threads (0: the hardware threads, at most 32) and builds
 * the element order, levels and CSRs on the device; its netlist is the
 * host reader's, and it hands every text the host reader rejects (and
 * netlists whose levels are not sorted in element order, and texts it
 * finds no device memory for) back to that reader, so errors and their
 * messages do not change.  Replaces the
 * istream parsing and Kahn sort of _read_graph (fsim/simulation.cpp:664-941). */
#define FSIMB_LOAD_AUTO 0
#define FSIMB_LOAD_HOST 1
#define FSIMB_LOAD_DEVICE 2
int fsimb_set_loader(fsimb_handle* h, int mode, int threads);

/* How the last circuit was loaded. */
typedef struct {
  uint32_t on_device;     /* 1: built by the device loader */
  uint32_t handed_back;   /* 1: the device loader handed the text to the host reader */
  uint32_t threads;       /* tokenizer threads (1 for the host reader) */
  uint32_t waves;         /* element-order waves: longest path from the PIs + 1 */
  double ms_total, ms_tokenize, ms_device;
} fsimb_load_info;
int fsimb_get_load_info(const fsimb_handle* h, fsimb_load_info* out);
/* Faults by topological index: pin 0 = output, k = k-th input; value 0/1.
 * Replaces _read_fault (fsim/simulation.cpp:943-959) for callers that hold
 * the list in memory; input-pin faults have no reference representation. */
int fsimb_set_faults(fsimb_handle* h, const uint32_t* site, const uint8_t* pin,
                     const uint8_t* value, uint64_t n);
int fsimb_set_fault_text(fsimb_handle* h, const char* flst, size_t flst_len);
/* Pattern words [ceil(P/64)][nPI], round-major (replaces _read_pattern). */
int fsimb_set_patterns(fsimb_handle* h, const uint64_t* words, uint64_t num_patterns);

/* Simulation.  Replaces Simulator::run(Mode, threads) (fsim/simulation.cpp:65-92)
 * and CUDAMAPartitioner::prepare_gpu_simulation()/run() (cuda_MA_partition.cu:496-538).
 * opts may be NULL.  The call returns after the results are on the host. */
int fsimb_run(fsimb_handle* h, const fsimb_opts* opts);

/* Results of the last run. */
int fsimb_results(const fsimb_handle* h, fsimb_fault_result* out, uint64_t n);
/* The reference's found_fault_to_pattern() view, 2 entries per fault
 * (fsim/simulation.hpp:89-91). */
int fsimb_found_fault_to_pattern(const fsimb_handle* h, uint64_t* out, uint64_t n);
/* Good-machine words of all N elements for one round, masked to the round's
 * valid bits; topological order [PIs, gates, POs].  After fsimb_run this is
 * g_pi/g_gate/g_po_results() of the reference for round = num_rounds-1
 * (fsim/simulation.hpp:57-59). */
int fsimb_good_values(const fsimb_handle* h, uint64_t round, uint64_t* out, uint64_t n);

/* Introspection (fsim/simulation.hpp:62-94). */
int fsimb_get_info(const fsimb_handle* h, fsimb_info* out);
int fsimb_get_stats(const fsimb_handle* h, fsimb_stats* out);
/* gate_idx_to_tpg_order_idx(): file id -> topological index, n = elements */
int fsimb_topo_map(const fsimb_handle* h, uint64_t* out, uint64_t n);
/* level of each element in topological order, n = elements */
int fsimb_levels(const fsimb_handle* h, uint64_t* out, uint64_t n);
/* num_gates_per_level(), n = num_levels */
int fsimb_gates_per_level(const fsimb_handle* h, uint64_t* out, uint64_t n);
/* gate types in topological order (GateType numbering; PI = 9, PO = 10) */
int fsimb_types(const fsimb_handle* h, uint8_t* out, uint64_t n);
/* loaded faults: topological site, pin, value */
int fsimb_faults(const fsimb_handle* h, uint32_t* site, uint8_t* pin, uint8_t* value, uint64_t n);
/* How faults share work, for splitting a fault list across GPUs (no
 * counterpart in the reference, which runs on one machine): group[f] names
 * the sweep fault f needs -- faults with equal groups share one (the faults
 * of one fanout-free region) -- and cost[f] estimates that group's work in
 * gate evaluations per pattern word (the same value for every fault of the
 * group).  Keep a group on one GPU and balance the groups' costs.  Works on
 * host-only handles; either pointer may be NULL; n = num_faults. */
int fsimb_fault_costs(fsimb_handle* h, uint64_t* group, uint64_t* cost, uint64_t n);
/* loaded pattern words, n = rounds * nPI */
int fsimb_patterns(const fsimb_handle* h, uint64_t* out, uint64_t n);
/* Graphviz DOT text of the loaded circuit in the layout of the reference's
 * Simulator::visualization_graph (fsim/simulation.cpp:1157-1236): fanin
 * edges of gates and POs inside cluster_0, then the PI and PO nodes.
 * Works on host-only handles.  Release the text with fsimb_free_text. */
int fsimb_dot(const fsimb_handle* h, char** text, size_t* len);

/* Good-machine PO words without allocating device memory.  This entry point
 * has no counterpart in the reference.  It serves callers that may not call
 * cudaMalloc/cudaFree (or any allocating routine) at this point: code that
 * runs under a device-memory budget fixed up front, or a serving loop that
 * cannot take the device-wide synchronisation those calls imply.
 *   d_pattern_words  device array [n_words][nPI], round-major like .ptn rows
 *   n_words          1..32 pattern words (up to 2048 patterns)
 *   d_po_words       device array [n_words][nPO]: good-machine PO words, not
 *                    masked to a partial round's valid bits
 * The element values live in one static device array that holds circuits of
 * up to 32,768 elements (8 MiB on every GPU that loads the library, kept until
 * the process exits); larger circuits fail with FSIMB_ERR_LIMIT.  The circuit
 * must already be on the device (after one fsimb_run on h).  The first call
 * on a device looks up the array's device address once: make that first call
 * before any stream capture.  All calls share the array and it keeps the last
 * call's contents; every value is written before it is read, so nothing needs
 * clearing, but calls whose kernels overlap on the GPU race on it.  Returns
 * after the kernels are enqueued on `stream` (NULL: the handle's stream).
 * The kernels wait for the uploads of the handle's last fsimb_run, whatever
 * stream it used; the caller orders what comes later on the handle (a run
 * after new faults or a new circuit replaces the arrays these kernels read)
 * after `stream`.  A device reset ends the handle and the looked-up address. */
int fsimb_good_po_noalloc(fsimb_handle* h, const uint64_t* d_pattern_words, uint32_t n_words,
                          uint64_t* d_po_words, void* stream);

/* ------------------------------------------------------------------ batches
 * Many circuits, each with its own fault list and pattern block, simulated
 * together.  No counterpart in the reference, whose drivers simulate one
 * circuit per process (main/simple.cpp:21-39, main/MA_partition.cu:40-63).
 * One run launches, for all members at once: the good machine one launch per
 * level index, the sweeps as one persistent launch per words-per-item class
 * pulling (circuit, tile, sweep, subtile) items from a device work counter,
 * and one launch each for FFR tracing and exact faults.  The sequence is
 * captured into a CUDA graph and replayed while the membership stays the same.
 * Members are handles loaded with circuit, faults and patterns; host-only
 * handles (device -1) are enough.  The batch borrows them until
 * fsimb_batch_clear or fsimb_batch_destroy and writes each member's results
 * into it (read them with fsimb_results / fsimb_found_fault_to_pattern);
 * they equal what fsimb_run gives in count mode.  Changing a member's inputs
 * between runs is allowed: the batch notices and lays out again. */
typedef struct fsimb_batch fsimb_batch;

typedef struct {
  uint32_t struct_size;
  uint32_t words_per_item;   /* 0 auto, or 1, 2, 4, 8 (members whose live values
                                do not fit take the next smaller value) */
  uint32_t block_threads;    /* 0 auto, or a multiple of 32 up to 1024 */
  uint32_t ctas_per_sm;      /* 0 auto (1), or 1..4: sizes the sweep CTA's record buffer */
  uint32_t tune;             /* 1, with the three above 0: time candidate shapes on a
                                sample of the batch (the first tile of a spread of its
                                circuits) the first time a membership runs; the winner
                                is kept until the membership changes */
  uint32_t no_graph;         /* 1: launch the kernels directly instead of through a graph */
  uint32_t reupload;         /* 1: copy every member's inputs (circuit, plan, patterns)
                                from host memory again even if none changed */
  uint32_t serial_classes;   /* 1: run the sweep classes one after another instead of
                                as concurrent branches */
  void* stream;              /* cudaStream_t; NULL: the batch's stream */
} fsimb_batch_opts;

typedef struct {
  double ms_total;           /* layout upload + kernels + result copies */
  double ms_h2d, ms_compute, ms_d2h;
  double ms_good, ms_sweep, ms_ffr;  /* phases, when run without the graph */
  double ms_tune;            /* autotuner time in this run (0 when reused) */
  double ms_host_prep;       /* host planning and scheduling in this run */
  uint64_t n_circuits, n_faults;
  uint64_t fault_patterns;   /* sum over members of faults x patterns */
  uint64_t sweep_items, ffr_units, exact_units, good_units;
  uint64_t dense_gate_words, sweep_alg_bytes, good_gate_words;
  uint64_t kernel_launches;  /* kernels in the launch sequence */
  uint32_t graph_used, n_classes;
  uint32_t words_per_item, block_threads, blocks, smem_bytes, ctas_per_sm;  /* largest class */
  uint32_t pad;
  uint64_t device_bytes;
  uint64_t h2d_bytes, d2h_bytes;  /* host<->device bytes copied by this run */
} fsimb_batch_stats;

int fsimb_batch_create(int device, fsimb_batch** out);
int fsimb_batch_destroy(fsimb_batch* b);
const char* fsimb_batch_last_error(const fsimb_batch* b);
int fsimb_batch_add(fsimb_batch* b, fsimb_handle* member);
int fsimb_batch_clear(fsimb_batch* b);
int fsimb_batch_size(const fsimb_batch* b, uint64_t* n);
int fsimb_batch_run(fsimb_batch* b, const fsimb_batch_opts* opts);
int fsimb_batch_get_stats(const fsimb_batch* b, fsimb_batch_stats* out);
/* Sweep classes of the last run: circuits sharing one sweep launch shape. */
typedef struct {
  uint32_t words_per_item, block_threads, blocks, smem_bytes;
  uint64_t n_circuits, sweep_items;
  uint32_t max_live, widest_level;
  double ms_sweep;           /* the class's launch, when run without the graph */
} fsimb_batch_class;
int fsimb_batch_class_stats(const fsimb_batch* b, uint32_t index, fsimb_batch_class* out);
/* Member indices (order of fsimb_batch_add) of a class; n >= its n_circuits. */
int fsimb_batch_class_members(const fsimb_batch* b, uint32_t index, uint32_t* out, uint64_t n);

/* ------------------------------------------------------------------ serving
 * A request loop over resident circuits.  No counterpart in the reference.
 * A circuit added to a server stays on the device with its sweep schedule
 * and, optionally, a resident block of patterns whose good-machine values
 * are computed once; a request names a fault subset and a range of those
 * patterns (or brings its own patterns).  Requests are submitted from any
 * thread and return a ticket at once; planner threads plan them, and a
 * dispatcher runs them in waves on `slots` concurrent slots, each with a
 * fixed device arena of `slot_bytes` allocated when the server starts: a
 * wave takes planned requests in ticket order while they fit its slot and
 * its predicted GPU time stays within `max_wave_ms`, so admission is by
 * device footprint, small requests are not held up behind large ones, and
 * serving allocates no device memory.
 * While one slot's wave runs, requests that arrive meanwhile are planned and
 * launched on the next free slot, and their work overlaps on the GPU.
 * A request's results equal fsimb_run's for the same circuit, faults and
 * patterns (count mode).  All fsimb_server_* calls are thread-safe. */
typedef struct fsimb_server fsimb_server;

typedef struct {
  uint32_t struct_size;
  uint32_t slots;             /* waves in flight at once: 0 -> 2, at most 8 */
  uint64_t slot_bytes;        /* device bytes of each slot's arena: 0 -> 4 GiB */
  uint32_t max_wave_requests; /* 0 -> 256 */
  uint32_t planner_threads;   /* host threads planning requests: 0 -> auto */
  uint32_t max_wave_ms;       /* a wave's predicted GPU time limit (a request that alone
                                 exceeds it runs alone): 0 -> 200 */
  uint32_t reserved;          /* 0 */
} fsimb_server_opts;

typedef struct {
  uint32_t struct_size;
  uint32_t circuit;           /* id from fsimb_server_add_circuit */
  const uint32_t* site;       /* faults by topological index (as fsimb_set_faults) */
  const uint8_t* pin;         /* NULL: output faults */
  const uint8_t* value;
  uint64_t n_faults;
  uint64_t n_patterns;        /* patterns of the request */
  uint64_t row0;              /* first row (64 patterns each) of the circuit's resident
                                 block, a multiple of 32; rows row0 .. row0 +
                                 ceil(n_patterns / 64) are the request's patterns */
  const uint64_t* words;      /* or the request's own words [ceil(P/64)][nPI]; then row0
                                 is ignored and its good machine runs in its wave */
} fsimb_request;

typedef struct {
  uint64_t completed, failed, waves, circuits;
  double mean_wave_requests;
  double fault_patterns;      /* sum over completed requests of faults x patterns */
  double wall_ms;             /* first submit to last completion since the reset */
  double ms_gpu_busy;         /* sum of wave durations on the GPU (overlapping waves both count) */
  double latency_p50_ms, latency_p99_ms, latency_mean_ms, latency_max_ms;  /* submit -> done */
  double queue_p50_ms, queue_p99_ms;      /* submit -> wave launch */
  double wave_gpu_p50_ms, wave_gpu_p99_ms;
  uint64_t resident_bytes;    /* device bytes of the resident circuits */
  uint64_t slot_bytes;        /* device bytes of the slots' arenas */
} fsimb_server_stats;

int fsimb_server_create(int device, const fsimb_server_opts* opts, fsimb_server** out);
/* Finishes the requests in flight, then frees everything. */
int fsimb_server_destroy(fsimb_server* s);
const char* fsimb_server_last_error(const fsimb_server* s);
/* Circuit text (.ckt) and an optional resident pattern block [ceil(P/64)][nPI].
 * Texts of 4 MiB and more are loaded by the device loader (fsimb_set_loader). */
int fsimb_server_add_circuit(fsimb_server* s, const char* ckt, size_t ckt_len, const uint64_t* words,
                             uint64_t n_patterns, uint32_t* id);
int fsimb_server_submit(fsimb_server* s, const fsimb_request* req, uint64_t* ticket);
/* Waits up to timeout_ms (< 0: no limit) for a ticket.  FSIMB_OK: the results
 * are in out[0..n) and the ticket is released; FSIMB_ERR_TIMEOUT: not done
 * yet; any other status: the request failed (message in last_error) and the
 * ticket is released. */
int fsimb_server_wait(fsimb_server* s, uint64_t ticket, fsimb_fault_result* out, uint64_t n,
                      int64_t timeout_ms);
int fsimb_server_get_stats(fsimb_server* s, fsimb_server_stats* out);
int fsimb_server_reset_stats(fsimb_server* s);

/* Synthetic workloads (seeded; text in LSIM's formats).  Returned buffers
 * are released with fsimb_free_text. */
typedef struct {
  uint32_t struct_size;
  uint64_t seed;
  uint32_t n_gates, n_pi, n_po, n_levels;
  uint32_t window;          /* inputs at most this many levels back (4) */
  double p_fanin3;          /* multi-input gates: P(3 inputs) */
  uint32_t type_mask;       /* bit t allows GateType t */
  double hub_frac;          /* fraction of gates with a large fanout target */
  uint32_t hub_fo_min, hub_fo_max, fo_min, fo_max;
  double p_unused;
  int32_t shuffle_ids;
} fsimb_gen_config;
int fsimb_gen_circuit(const fsimb_gen_config* cfg, char** text, size_t* len);
/* Fault list for a circuit given as .ckt text.  kind 0: every gate output
 * SA0/SA1 (plain .flst); 1: outputs and input pins; 2: outputs and input pins
 * collapsed by equivalence (pin lists use the "@pins" .flst form). */
int fsimb_gen_faults(const char* ckt, size_t ckt_len, int kind, char** text, size_t* len);
int fsimb_gen_patterns(uint64_t seed, uint64_t n_patterns, uint64_t n_pi, double biased_pi_frac,
                       double p_one_biased, char** text, size_t* len);
void fsimb_free_text(char* text);

#ifdef __cplusplus
}
#endif

#endif /* FSIMB_H */
