"""Benchmark: fault x pattern evaluations per second on the 200k-gate workload.

Workload (c2, lsim_b200/gen.py): seeded synthetic circuit with 200,000 gates,
1,000 PIs, 1,000 POs and 150 levels (mean fan-in 2.2); SA0/SA1 on every gate
output and input pin, collapsed by equivalence; 65,536 uniform patterns.
One step simulates every fault against every pattern (count mode) and brings
the per-fault results back to the host.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value: device time of K steps with circuit, faults and patterns resident on
the GPU (CUDA events on the launch stream, max over ranks).
e2e:   the same through the public API from host buffers: pattern words
       uploaded from pinned host memory and per-fault results read back every
       step.
With N > 1 each rank simulates its own 65,536-pattern block (seed = rank)
and the per-fault results are merged across ranks every step (weak scaling);
with --shard faults each rank simulates its part of the fault list (whole
fanout-free-region groups, balanced by estimated cost) over the same
patterns, merged the same way (strong scaling).
--impl reference times LSIM's own CPU simulator (oracle/_ref, else the CPU
port in oracle/) on a bounded sample of the same workload on all host cores;
its inputs come from the pure-Python generator (tests/workload_py.py), so
that process loads no library of this package.  Both arms print the same
config.

The default line also carries: gate-word evaluations per second; an HBM
roofline (compulsory DRAM bytes of a sweep launch over its time) and the
on-chip one that binds the sweep (operand bytes through shared memory);
the reference's other CPU modes and the oracle's cone-limited restatement
(cpu_baselines_other); and, at N = 1, the batched (c4, 2 steps) and served
(c5, burst and one Poisson rate) summaries (--no-extras leaves them out).

--workload c4 times the batched configuration instead: 256 circuits
(gen.batch_configs: 500-50,000 gates log-uniform, 10-120 levels, SA0/SA1 on
every gate output, 1,024-16,384 patterns) run as one batch (fsimb_batch_*,
CUDA graph, autotuned sweep shape) against the same 256 circuits run one
after another through the plain per-circuit path, both with inputs resident
(value) and with every input copied from host memory each step (e2e).
--gates LO,HI changes the gate-count range (e.g. 500,5000 for many circuits
that are each too small to fill the GPU).

--workload c5 times the serving configuration: 32 resident circuits
(gen.serve_configs: 1,000-500,000 gates), requests of 1,000-100,000 faults
and 64-8,192 patterns served by the server (fsimb_server_*) and by the plain
path one job at a time, all at once and at Poisson arrival rates; it reports
p50/p99 latency and fault-patterns/s for both.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "c2"
METRIC = "fault×pattern evals/s (200k-gate)"
UNIT = "fault-patterns/s"
# The c2 workload's fixed sizes (seeded; checked against the loaded problem
# in the GPU arm, so both arms print the same config).
C2_FAULTS = 738943
C2_PATTERNS = 65536
C2_ELEMENTS = 202000
# Shared-memory bandwidth of one SM: 32 banks x 4 bytes per clock.
SMEM_BYTES_PER_CLK_SM = 128


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback (6.65 TB/s, an earlier copy measurement on this pool)"


def _profile_summary():
    """Per-launch DRAM bytes and on-chip counters of the sweep kernel from
    the committed ncu summaries (key: value lines)."""
    out = {}
    for name in ("k_sweep_c2.md", "k_sweep_c2s.md"):
        try:
            for line in open(os.path.join(ROOT, "profiles", name)):
                if ":" in line and line.split(":", 1)[0].strip().startswith(("traffic_", "ncu_")):
                    k, v = line.split(":", 1)
                    try:
                        out[k.strip()] = float(v)
                    except ValueError:
                        pass
        except OSError:
            pass
    return out


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        self.gpu = vis.split(",")[local_rank] if vis else str(local_rank)
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-i", self.gpu, "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().splitlines() if r.count(",") >= 8]
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(rows)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _config(world, faults_sharded):
    """The workload as both arms state it."""
    patterns = C2_PATTERNS if (faults_sharded or world == 1) else world * C2_PATTERNS
    return {"workload": "c2: 200,000 gates, 1,000 PI, 1,000 PO, 150 levels, mean fan-in 2.2; "
                        "%d collapsed output+input-pin SA faults; 65,536 patterns%s"
                        % (C2_FAULTS, "" if patterns == C2_PATTERNS else
                           " per rank (%d ranks, own seed each)" % world),
            "faults": C2_FAULTS, "patterns": patterns, "elements": C2_ELEMENTS, "mode": "count",
            "parallelism": ("1 GPU" if world == 1 else
                            "%s-sharded x%d" % ("fault" if faults_sharded else "pattern", world)),
            "l2": "inputs larger than L2: the good-machine words (1.65 GB per 65,536-pattern "
                  "block) are rewritten every step"}


def _ref_threads():
    return max(1, min(64, os.cpu_count() or 1))


def reference_sample(target_s=15.0, inputs=None):
    """LSIM's own simulator (oracle/_ref; the CPU port in oracle/ when the
    reference was not built) on a bounded sample of the c2 workload: its
    first 4 x threads output faults (the reference's .flst cannot express
    pin faults) over as many 64-pattern rounds as fit in about target_s,
    faults sharded over all host threads.  Inputs come from the pure-Python
    generator (tests/workload_py.py), so nothing of the product library is
    loaded.  Returns (cpu_baseline dict, inputs)."""
    from tests.oracle_lib import Oracle, Reference, ref_available
    from tests import workload_py
    threads = _ref_threads()
    kind = "reference" if ref_available() else "port"
    nf = 4 * threads if kind == "reference" else 32 * threads
    if inputs is None or inputs["flst"].count("\n") - 1 < nf:
        inputs = workload_py.c2_inputs(rounds=1024, n_output_faults=nf)
    words, n_pi = inputs["words"], inputs["n_pi"]

    def run(R):
        w = words[:R]
        if kind == "reference":
            ref = Reference(inputs["ckt"], inputs["flst"], words=w, P=R * 64, n_pi=n_pi)
            ref.simulate(threads=threads)
            return ref.seconds, ref.F
        o = Oracle(inputs["ckt"], inputs["flst"], "0\n")
        o.set_patterns(w, R * 64)
        t0 = time.perf_counter()
        o.simulate(mode=0, threads=threads)
        return time.perf_counter() - t0, len(o.faults)

    per_round, _ = run(1)
    R = int(max(1, min(len(words), target_s / max(per_round, 1e-3))))
    secs, F = run(R)
    value = F * R * 64 / secs
    return ({"value": value, "unit": UNIT, "cores": threads, "kind": kind, "cpu": _cpu_model(),
             "sample": "%d output faults x %d rounds (%d patterns) of the c2 workload, %.1f s, "
                       "faults sharded over %d threads (full re-simulation per fault, "
                       "fsim/simulation.cpp:104-147)" % (F, R, R * 64, secs, threads)}, inputs)


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def extra_cpu_baselines(c2_text=None):
    """The reference's other CPU modes and the oracle's cone-limited
    restatement, each on a bounded sample (a few seconds each)."""
    from tests.oracle_lib import Oracle, Reference, ref_available
    from tests import workload_py
    out = []
    threads = _ref_threads()
    if ref_available():
        c1 = dict(n_gates=2000, n_pi=64, n_po=64, n_levels=30, p_fanin3=0.5, seed=0)
        ckt = workload_py.circuit(**c1)
        words = workload_py.pattern_words(64, 4096, seed=0)
        nf = 128
        # SA0/SA1 on the first 64 gates by file id (c1's list is every gate output)
        flst = "%d\n%s\n" % (nf, "\n".join("%d %d" % (128 + i // 2, i % 2) for i in range(nf)))
        for mode, name, th in ((0, "SEQUENTIAL", 1), (2, "PARALLEL_OMP", threads),
                               (1, "PARALLEL_TF", threads)):
            ref = Reference(ckt, flst, words=words, P=4096, n_pi=64)
            t0 = time.perf_counter()
            ref.run_table(mode=mode, threads=th)
            secs = time.perf_counter() - t0
            out.append({"value": nf * 4096 / secs, "unit": UNIT, "cores": th, "kind": "reference",
                        "mode": name, "cpu": _cpu_model(),
                        "sample": "c1 (2,000 gates, 64 PI / 64 PO, 30 levels), %d output faults x "
                                  "4,096 patterns through Simulator::run(%s, %d) "
                                  "(fsim/simulation.cpp:65-92), %.2f s" % (nf, name, th, secs)})
    if c2_text is not None:
        # every 512th fault of the whole collapsed list (output and pin faults)
        sel = np.arange(0, c2_text["n_faults"], 512)
        fl = workload_py.flst_pins(c2_text["fault_fids"][sel], c2_text["fault_pins"][sel],
                                   c2_text["fault_values"][sel])
        R = min(64, len(c2_text["words"]))
        o = Oracle(c2_text["ckt"], fl, "0\n")
        o.set_patterns(c2_text["words"][:R], R * 64)
        t0 = time.perf_counter()
        o.simulate(mode=2, threads=threads)
        secs = time.perf_counter() - t0
        F = len(o.faults)
        out.append({"value": F * R * 64 / secs, "unit": UNIT, "cores": threads, "kind": "port",
                    "mode": "cone-limited restatement over chunks of rounds "
                            "(oracle/fsim_oracle.c mode 2)",
                    "cpu": _cpu_model(),
                    "sample": "c2, every 512th fault of the collapsed list (%d output and pin "
                              "faults) x %d rounds, %.2f s" % (F, R, secs)})
    return out


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return
    faults_sharded = args.shard == "faults"
    cfg = _config(world, faults_sharded)
    units = C2_FAULTS * cfg["patterns"]
    # each step a bounded sample sized so that the whole run takes a few minutes
    per_step = max(2.0, min(args.ref_seconds, 150.0 / max(1, args.steps + args.warmup)))
    inputs = None
    for _ in range(args.warmup):
        _, inputs = reference_sample(target_s=min(2.0, per_step), inputs=inputs)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        b, inputs = reference_sample(target_s=per_step, inputs=inputs)
        vals.append(b["value"])
    elapsed = time.perf_counter() - t0
    value = statistics.median(vals)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * units / value,
            "higher_is_better": True, "scaling": "strong" if faults_sharded else "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic", "impl": "reference",
            "config": cfg,
            "timed": "each step is a bounded sample of the workload (output faults x rounds, "
                     "see cpu_baseline.sample); ms_per_step is the full job at the sample's rate",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": b["cores"], "kind": b["kind"],
                             "cpu": b["cpu"], "sample": b["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": elapsed}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from lsim_b200 import Simulator, gen, shard

    faults_sharded = args.shard == "faults"
    # pattern sharding: each rank its own 65,536-pattern block (weak scaling);
    # fault sharding: one block, each rank its part of the fault list (strong)
    w = gen.workload(WORKLOAD, pattern_seed=0 if faults_sharded else rank)
    sim = Simulator(local)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    F_all = sim.info().num_faults
    if F_all != C2_FAULTS or sim.info().num_elements != C2_ELEMENTS:
        raise RuntimeError("the c2 workload changed: %d faults, %d elements"
                           % (F_all, sim.info().num_elements))
    my_faults = None
    if faults_sharded and world > 1:
        site, pin, val = sim.faults()
        group, cost = sim.fault_costs()
        my_faults = shard.split_faults(group, cost, world)[rank]
        sim.set_faults(site[my_faults], pin[my_faults], val[my_faults])
    info = sim.info()
    F, P = info.num_faults, info.num_patterns
    words = sim.patterns()
    pinned = torch.from_numpy(words.ravel()).pin_memory()
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    def merge(res):
        if world == 1:
            return res
        # rank 0 reports: the parts are gathered (fault shards) or reduced
        # (pattern shards) onto it only
        if faults_sharded:
            return shard.merge_fault_shards(res, my_faults, F_all, info.num_rounds, device="cuda",
                                            dst=0)
        return shard.merge_results(res, rank * P, rank == world - 1, world * info.num_rounds,
                                   device="cuda", dst=0)

    tune_ms = 0.0
    for _ in range(args.warmup):
        sim.run(stream=sp, tune=True)  # the first run tunes the sweep shape
        tune_ms += sim.stats()["ms_tune"]
        merge(sim.results())
    torch.cuda.synchronize()

    # value: inputs resident, K steps
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sweep_ms, sweep_bytes, tiles, launches, gwe, good_gwe = 0.0, 0, 0, 0, 0, 0
    for _ in range(args.steps):
        sim.run(stream=sp, tune=True)
        merged = merge(sim.results())
        st = sim.stats()
        sweep_ms += st["ms_sweep"]
        sweep_bytes += st["sweep_alg_bytes"]
        tiles += st["n_tiles"]
        launches += st["kernel_launches"]
        gwe += st["dense_gate_words"]
        good_gwe += st["good_gate_words"]
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if dist:
        dist.barrier()
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # e2e: patterns from pinned host memory each step, results back each step
    host_words = pinned.numpy()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(args.steps):
        sim.set_patterns(host_words, P)
        sim.run(stream=sp, tune=True)
        merged = merge(sim.results())
    g1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = g0.elapsed_time(g1)
    if dist:
        t = torch.tensor([ms_e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    del merged

    units = (float(F_all) if faults_sharded else float(world) * F) * P * args.steps
    value = units / (ms / 1e3)
    e2e = units / (ms_e2e / 1e3)
    st = sim.stats()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if faults_sharded else "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic", "config": _config(world, faults_sharded),
        "e2e": {"value": e2e, "unit": UNIT,
                "h2d_bytes_per_step": int(words.nbytes),
                "d2h_bytes_per_step": int(F * 17)},
        "gpu_launches": int(launches),
        "gate_word_evals_per_s": {
            "sweep_dense": gwe / (ms / 1e3) * (world if not faults_sharded else 1),
            "good_machine": good_gwe / (ms / 1e3) * (world if not faults_sharded else 1),
            "per_step_sweep": gwe / args.steps,
            "definition": "one gate evaluated on one 64-pattern word; the sweeps evaluate every "
                          "gate above the flipped element's level (dense), per sweep and word"},
        "sweep": {"words_per_item": st["words_per_item"], "block_threads": st["block_threads"],
                  "blocks": st["blocks"], "ctas_per_sm": st["ctas_per_sm"],
                  "smem_bytes": st["smem_bytes"], "max_live": st["max_live"],
                  "shape": "autotuned during warm-up on a strided sample of the first tile's "
                           "sweeps", "tune_ms": tune_ms},
        "breakdown_ms_per_step": {"good": st["ms_good"], "sweep": st["ms_sweep"],
                                  "ffr": st["ms_ffr"], "compute": st["ms_compute"],
                                  "total": st["ms_total"]},
        "clocks": clk,
    }
    line.update(_rooflines(sweep_ms / max(1, tiles) / 1e3, sweep_bytes / max(1, tiles),
                           st, clk))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        b, inputs = reference_sample(target_s=args.ref_seconds)
        line["cpu_baseline"] = b
        line["cpu_baselines_other"] = extra_cpu_baselines(inputs)
    sim.close()
    if rank == 0 and world == 1 and not args.no_extras:
        line["batched"] = batch_summary(args.extra_circuits, steps=2)
        line["served"] = serve_summary(n_req=args.requests, rates=[1.0])
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _rooflines(launch_s, alg_bytes, st, clk):
    """HBM roofline of the sweep kernel from its compulsory DRAM bytes, and
    the on-chip roofline that binds it (shared-memory bandwidth)."""
    peak, peak_src = _peaks()
    prof = _profile_summary()
    traffic = prof.get("traffic_per_launch_bytes")
    # compulsory DRAM bytes of one launch: the tile's good words, the gate
    # records and live-in lists of the schedule, the sweep output rows
    compulsory = st["hbm_bytes_per_tile"]
    hbm = compulsory / launch_s / 1e9 if launch_s > 0 else 0.0
    mhz = (clk or {}).get("sm_mhz") or 1965.0
    smem_peak = SMEM_BYTES_PER_CLK_SM * 148 * mhz * 1e6 / 1e9
    onchip = alg_bytes / launch_s / 1e9 if launch_s > 0 else 0.0
    return {
        "roofline": {"bound": "hbm", "achieved": hbm, "peak": peak, "unit": "GB/s",
                     "frac": hbm / peak, "traffic": traffic, "kernel": "k_sweep",
                     "peak_source": peak_src,
                     "per_launch_bytes": compulsory, "per_launch_ms": launch_s * 1e3,
                     "note": "achieved = compulsory DRAM bytes of one launch (good words of the "
                             "tile, gate records, live-in lists, output rows) / its CUDA-event "
                             "time; traffic = ncu dram bytes of one launch. Values stay in "
                             "shared memory, so HBM is not what binds this kernel (see onchip)"},
        "onchip": {"bound": "shared-memory bandwidth", "achieved": onchip, "peak": smem_peak,
                   "unit": "GB/s", "frac": onchip / smem_peak,
                   "peak_source": "architectural: 128 B/clock/SM x 148 SMs x the median SM clock "
                                  "sampled during the timed region (%.0f MHz)" % mhz,
                   "per_launch_alg_bytes": alg_bytes,
                   "achieved_definition": "8*(fanin+1) bytes per gate-word evaluation: the "
                                          "fanin words read and the output word written, all "
                                          "in shared memory",
                   "ncu": {k[4:]: v for k, v in prof.items() if k.startswith("ncu_")}},
    }


def run_batch(args):
    """Batched configuration: one batch of 256 circuits against 256 plain runs."""
    lo, hi = (int(x) for x in args.gates.split(","))
    print(json.dumps(batch_measure(args.circuits, args.steps, args.warmup, gates=(lo, hi))), flush=True)


def batch_summary(n_circuits, steps=2):
    """The batched configuration's figures for the default bench line."""
    m = batch_measure(n_circuits, steps, warmup=1, full=False)
    return {"workload": m["config"]["workload"], "steps": steps, "value": m["value"],
            "unit": UNIT, "ms_per_step": m["ms_per_step"], "plain_sequential": m["plain_sequential"],
            "batch_over_plain": m["batch_over_plain"], "e2e": m["e2e"],
            "plain_sequential_e2e": m["plain_sequential_e2e"], "gpu_launches": m["gpu_launches"],
            "n_classes": m["config"]["sweep"]["n_classes"], "graph": m["config"]["graph"],
            "tune_ms": m["config"]["tune_ms"], "results_equal_plain": m["results_equal_plain"],
            "clocks": m["clocks"]}


def batch_measure(n_circuits, steps, warmup, full=True, gates=(500, 50000)):
    import torch
    from lsim_b200 import Batch, Simulator, gen
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    cfgs = gen.batch_configs(n_circuits, seed=0, gates=gates)
    t0 = time.perf_counter()
    ws = [gen.generate(**c) for c in cfgs]
    gen_s = time.perf_counter() - t0
    members, plains = [], []
    for w in ws:
        m = Simulator(-1)
        m.read_text(w["ckt"], w["flst"], w["ptn"])
        members.append(m)
        p = Simulator(0)
        p.read_text(w["ckt"], w["flst"], w["ptn"])
        plains.append(p)
    F = sum(m.info().num_faults for m in members)
    FP = sum(m.info().num_faults * m.info().num_patterns for m in members)
    gates = [c["n_gates"] for c in cfgs]
    b = Batch(0)
    for m in members:
        b.add(m)

    def timed(fn, steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    # warm-up: the first batch run tunes the sweep shape and captures the graph
    t0 = time.perf_counter()
    b.run(tune=True, stream=sp)
    first_s = time.perf_counter() - t0
    tune_ms = b.stats()["ms_tune"]
    for _ in range(max(0, warmup - 1)):
        b.run(tune=True, stream=sp)
    for p in plains:
        p.run(stream=sp, tune=True)
    clocks = ClockSampler(0)
    clocks.start()
    ms_batch = timed(lambda: b.run(tune=True, stream=sp), steps)
    st = b.stats()
    ms_serial = timed(lambda: b.run(tune=True, concurrent=False, stream=sp), steps) if full else None
    ms_plain = timed(lambda: [p.run(stream=sp, tune=True) for p in plains], steps)
    clk = clocks.stop()
    plain_launches = sum(p.stats()["kernel_launches"] for p in plains)
    # e2e: every input from host memory each step
    ms_batch_e2e = timed(lambda: b.run(tune=True, reupload=True, stream=sp), steps)
    st_e2e = b.stats()
    words = [p.patterns() for p in plains]
    pinned = [torch.from_numpy(wd.ravel()).pin_memory().numpy() for wd in words]

    def plain_e2e():
        for p, wd, m in zip(plains, pinned, members):
            p.set_patterns(wd, m.info().num_patterns)
            p.run(stream=sp, tune=True)
            p.results()
    ms_plain_e2e = timed(plain_e2e, steps)
    phases, classes = None, None
    if full:
        # phase split of one step of each arm (batch without the graph)
        b.run(tune=True, graph=False, stream=sp)
        st_ng = b.stats()
        classes = b.classes()
        phases = {"batch": {k: st_ng[k] for k in ("ms_good", "ms_sweep", "ms_ffr", "ms_total")},
                  "plain": {k: sum(p.stats()[k] for p in plains)
                            for k in ("ms_good", "ms_sweep", "ms_ffr", "ms_total")}}
    # results agree with the plain path on every circuit
    same = all(np.array_equal(m.results(), p.results()) for m, p in zip(members, plains))
    line = {
        "metric": "fault×pattern evals/s (batched, %d circuits)" % n_circuits,
        "value": FP * steps / (ms_batch / 1e3), "unit": UNIT, "n_gpus": 1,
        "steps": steps, "warmup": warmup, "ms_per_step": ms_batch / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic",
        "config": {"workload": "c4: %d circuits, %d-%d gates (median %d), 10-120 levels, SA0/SA1 "
                               "on every gate output (%d faults), 1,024-16,384 patterns"
                               % (n_circuits, min(gates), max(gates), int(np.median(gates)), F),
                   "fault_patterns_per_step": FP, "mode": "count",
                   "sweep": {k: st[k] for k in ("words_per_item", "block_threads", "ctas_per_sm",
                                                "blocks", "smem_bytes", "n_classes")},
                   "graph": bool(st["graph_used"]), "tune_ms": tune_ms,
                   "first_run_s": first_s, "generate_s": gen_s},
        "plain_sequential": {"value": FP * steps / (ms_plain / 1e3),
                             "ms_per_step": ms_plain / steps,
                             "gpu_launches_per_step": int(plain_launches)},
        "batch_over_plain": ms_plain / ms_batch,
        "e2e": {"value": FP * steps / (ms_batch_e2e / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": int(st_e2e["h2d_bytes"]),
                "d2h_bytes_per_step": int(st_e2e["d2h_bytes"])},
        "plain_sequential_e2e": {"value": FP * steps / (ms_plain_e2e / 1e3),
                                 "ms_per_step": ms_plain_e2e / steps},
        "gpu_launches": int(st["kernel_launches"]) * steps,
        "breakdown_ms_per_step": {"compute": st["ms_compute"], "d2h": st["ms_d2h"],
                                  "total": st["ms_total"]},
        "gate_word_evals_per_s": {"sweep_dense": st["dense_gate_words"] / (ms_batch / steps / 1e3)},
        "results_equal_plain": same,
        "clocks": clk,
    }
    if full:
        line["batch_serial_classes"] = {"value": FP * steps / (ms_serial / 1e3),
                                        "ms_per_step": ms_serial / steps}
        line["phases_ms_per_step"] = phases
        line["classes"] = classes
    b.close()
    for m in members + plains:
        m.close()
    return line


def run_serve(args):
    """Serving configuration: requests against 32 resident circuits, served
    by the server (waves on concurrent slots) and by the plain path one job
    at a time, at a burst and at Poisson arrival rates."""
    n_circ = args.circuits if args.circuits != 256 else 32
    print(json.dumps(serve_measure(n_circ, args.requests, args.rates, args.slots, args.slot_gib)),
          flush=True)


def serve_summary(n_req=200, rates=(1.0,), n_circuits=32):
    """The serving configuration's figures for the default bench line."""
    m = serve_measure(n_circuits, n_req, list(rates), 2, 8)
    return {"workload": m["config"]["workload"], "unit": UNIT, "burst": m["burst"],
            "poisson": m["poisson"], "rates": m["config"]["rates"],
            "results_equal_plain": m["results_equal_plain"], "clocks": m["clocks"]}


def serve_measure(n_circuits, n_req, rates, slots, slot_gib):
    import threading
    import torch
    from lsim_b200 import Server, Simulator, gen
    torch.cuda.set_device(0)
    rng = np.random.default_rng(0)
    cfgs = gen.serve_configs(n_circuits, seed=0)
    block_P = 16384
    circs = []
    t0 = time.perf_counter()
    for c in cfgs:
        ckt = gen.circuit(c["n_gates"], c["n_pi"], c["n_po"], c["n_levels"], p_fanin3=c["p_fanin3"],
                          seed=c["seed"])
        flst = gen.faults(ckt, c["faults"])
        ptn = gen.patterns(c["n_pi"], block_P, seed=c["seed"])
        h = Simulator(-1)
        h.read_text(ckt, flst, ptn)
        site, pin, val = h.faults()
        circs.append(dict(ckt=ckt, words=h.patterns(), site=site, pin=pin, value=val,
                          gates=c["n_gates"]))
    gen_s = time.perf_counter() - t0
    # the request stream: circuit, fault subset (1,000-100,000, log-uniform,
    # at most the circuit's list), 64-8,192 patterns from a tile-aligned window
    reqs = []
    for _ in range(n_req):
        ci = int(rng.integers(len(circs)))
        c = circs[ci]
        F = len(c["site"])
        k = min(F, int(round(np.exp(rng.uniform(np.log(1000), np.log(100000))))))
        idx = np.sort(rng.choice(F, size=k, replace=False))
        P = int(rng.integers(64, 8193))
        W = (P + 63) // 64
        row0 = 32 * int(rng.integers(0, (256 - W) // 32 + 1))
        reqs.append(dict(circuit=ci, site=c["site"][idx].copy(), pin=c["pin"][idx].copy(),
                         value=c["value"][idx].copy(), P=P, row0=row0))
    FP = sum(len(r["site"]) * r["P"] for r in reqs)

    srv = Server(0, slots=slots, slot_bytes=slot_gib << 30)
    t0 = time.perf_counter()
    ids = [srv.add_circuit(c["ckt"], c["words"], block_P) for c in circs]
    add_s = time.perf_counter() - t0
    plains = []
    for c in circs:
        p = Simulator(0)
        p.load_circuit(c["ckt"])
        plains.append(p)

    def serve_at(rate):
        """rate = requests/s (None: all at once); returns latency quantiles."""
        srv.reset_stats()
        arrivals = np.zeros(n_req) if rate is None else np.cumsum(rng.exponential(1.0 / rate, n_req))
        tickets = [None] * n_req
        start = time.perf_counter() + 0.05

        def client():
            for i, r in enumerate(reqs):
                d = start + arrivals[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets[i] = srv.submit(ids[r["circuit"]], r["site"], r["value"], pin=r["pin"],
                                        n_patterns=r["P"], row0=r["row0"])
        th = threading.Thread(target=client)
        th.start()
        th.join()
        for t in tickets:
            srv.wait(t)
        st = srv.stats()
        return {"rate_req_s": rate, "p50_ms": st["latency_p50_ms"], "p99_ms": st["latency_p99_ms"],
                "mean_ms": st["latency_mean_ms"], "value": st["fault_patterns"] / (st["wall_ms"] / 1e3),
                "waves": st["waves"], "mean_wave_requests": st["mean_wave_requests"],
                "wall_ms": st["wall_ms"], "gpu_wave_ms_sum": st["ms_gpu_busy"]}

    def plain_at(rate):
        arrivals = np.zeros(n_req) if rate is None else np.cumsum(rng.exponential(1.0 / rate, n_req))
        lat = []
        start = time.perf_counter() + 0.05
        for i, r in enumerate(reqs):
            d = start + arrivals[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            p = plains[r["circuit"]]
            c = circs[r["circuit"]]
            W = (r["P"] + 63) // 64
            p.set_faults(r["site"], r["pin"], r["value"])
            p.set_patterns(c["words"][r["row0"]:r["row0"] + W], r["P"])
            p.run()
            p.results()
            lat.append((time.perf_counter() - (start + arrivals[i])) * 1e3)
        wall = time.perf_counter() - start
        lat = np.array(lat)
        return {"rate_req_s": rate, "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                "value": FP / wall}

    # warm-up: one pass of the stream through each path
    serve_at(None)
    plain_at(None)
    clocks = ClockSampler(0)
    clocks.start()
    burst_srv = serve_at(None)
    burst_plain = plain_at(None)
    cap = n_req / (FP / burst_plain["value"])  # plain path capacity, requests/s
    rows = []
    for f in rates:
        rows.append({"load": f, "server": serve_at(f * cap), "plain": plain_at(f * cap)})
    clk = clocks.stop()
    # results of the mix equal the plain path's, request by request
    same = True
    for i in range(0, n_req, max(1, n_req // 16)):
        r = reqs[i]
        t = srv.submit(ids[r["circuit"]], r["site"], r["value"], pin=r["pin"], n_patterns=r["P"],
                       row0=r["row0"])
        got = srv.wait(t)
        p = plains[r["circuit"]]
        W = (r["P"] + 63) // 64
        p.set_faults(r["site"], r["pin"], r["value"])
        p.set_patterns(circs[r["circuit"]]["words"][r["row0"]:r["row0"] + W], r["P"])
        p.run()
        same &= bool(np.array_equal(got, p.results()))
    st = srv.stats()
    gates = [c["gates"] for c in circs]
    line = {
        "metric": "served fault×pattern evals/s with p50/p99 latency (32 resident circuits)",
        "value": burst_srv["value"], "unit": UNIT, "n_gpus": 1, "steps": n_req, "warmup": n_req,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic",
        "config": {"workload": "c5: %d resident circuits of %d-%d gates (median %d), %d-pattern "
                               "resident blocks; %d requests of 1,000-100,000 faults and 64-8,192 "
                               "patterns" % (len(circs), min(gates), max(gates),
                                             int(np.median(gates)), block_P, n_req),
                   "fault_patterns": FP, "slots": slots, "slot_gib": slot_gib,
                   "generate_s": gen_s, "add_circuits_s": add_s,
                   "resident_bytes": st["resident_bytes"], "slot_bytes": st["slot_bytes"],
                   "rates": "fractions of the plain path's burst capacity (%.2f requests/s)" % cap},
        "burst": {"server": burst_srv, "plain": burst_plain},
        "poisson": rows,
        "results_equal_plain": same,
        "clocks": clk,
    }
    srv.close()
    for p in plains:
        p.close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="leave the batched (c4) and served (c5) summaries out of the c2 line")
    ap.add_argument("--extra-circuits", type=int, default=256,
                    help="circuits of the batched summary in the c2 line")
    ap.add_argument("--workload", default=WORKLOAD, help="c2 (default) or another gen.WORKLOADS key")
    ap.add_argument("--shard", default="patterns", choices=["patterns", "faults"],
                    help="with --gpus N > 1: each rank its own pattern block (weak scaling, "
                         "default) or its part of the fault list (strong scaling)")
    ap.add_argument("--circuits", type=int, default=256,
                    help="circuits for --workload c4 (default 256) or c5 (default 32)")
    ap.add_argument("--gates", default="500,50000",
                    help="--workload c4: gate-count range of the circuits, log-uniform")
    ap.add_argument("--requests", type=int, default=200, help="requests for --workload c5")
    ap.add_argument("--rates", type=float, nargs="*", default=[0.5, 1.0, 2.0, 4.0],
                    help="--workload c5 Poisson rates, as fractions of the plain path's capacity")
    ap.add_argument("--slots", type=int, default=2, help="server slots for --workload c5")
    ap.add_argument("--slot-gib", type=int, default=8, help="server slot arena GiB for c5")
    ap.add_argument("--shape", default="",
                    help="with --profile: sweep shape 'words_per_item,block_threads,ctas_per_sm' "
                         "(the one the bench's tuner chose), else the default shape")
    ap.add_argument("--drop", action="store_true", help="with --profile: fault dropping")
    ap.add_argument("--profile", action="store_true",
                    help="one untimed run of the workload (for profiler captures)")
    args = ap.parse_args()
    if args.profile and args.workload == "c4":
        # one batch of the batched configuration's first --circuits circuits,
        # kernels launched directly (not through the graph)
        from lsim_b200 import Batch, Simulator, gen
        sims = []
        for c in gen.batch_configs(args.circuits, seed=0):
            w = gen.generate(**c)
            s = Simulator(-1)
            s.read_text(w["ckt"], w["flst"], w["ptn"])
            sims.append(s)
        b = Batch(0)
        for s in sims:
            b.add(s)
        for _ in range(max(1, args.steps)):
            b.run(graph=False)
        print(json.dumps({"workload": "c4", "circuits": args.circuits, "stats": b.stats(),
                          "classes": b.classes()}))
        b.close()
        return
    if args.profile:
        from lsim_b200 import Simulator, gen
        if args.workload == "c3":
            # the stated stress list: the collapsed output + input-pin faults of
            # the 2M-gate circuit, 4,000,000 of them drawn with seed 0
            w = gen.workload("c3", faults="collapsed")
        else:
            w = gen.workload(args.workload)
        sim = Simulator(0)
        sim.read_text(w["ckt"], w["flst"], w["ptn"])
        if args.workload == "c3":
            site, pin, val = sim.faults()
            keep = np.sort(np.random.default_rng(0).choice(len(site), size=4000000, replace=False))
            sim.set_faults(site[keep], pin[keep], val[keep])
        shape = {}
        if args.shape:
            M, T, occ = (int(x) for x in args.shape.split(","))
            shape = dict(words_per_item=M, block_threads=T, ctas_per_sm=occ)
        t0 = time.perf_counter()
        for _ in range(max(1, args.steps)):
            sim.run(drop=args.drop, **shape)
        wall = time.perf_counter() - t0
        st = sim.stats()
        res = sim.results()
        info = sim.info()
        print(json.dumps({"workload": args.workload, "faults": info.num_faults,
                          "pin_faults": int((sim.faults()[1] > 0).sum()),
                          "patterns": info.num_patterns, "elements": info.num_elements,
                          "mode": "drop" if args.drop else "count", "wall_s": wall,
                          "detected": int(res["detected"].sum()),
                          "gate_word_evals_per_s": st["dense_gate_words"] / max(st["ms_sweep"], 1e-9) * 1e3,
                          "stats": st}))
        return
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c4":
        run_batch(args)
    elif args.workload == "c5":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
