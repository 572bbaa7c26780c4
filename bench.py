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
port in oracle/) on a bounded sample of the same workload on all host cores.

--workload c4 times the batched configuration instead: 256 circuits
(gen.batch_configs: 500-50,000 gates log-uniform, 10-120 levels, SA0/SA1 on
every gate output, 1,024-16,384 patterns) run as one batch (fsimb_batch_*,
CUDA graph, autotuned sweep shape) against the same 256 circuits run one
after another through the plain per-circuit path, both with inputs resident
(value) and with every input copied from host memory each step (e2e).

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


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic():
    """Per-launch DRAM bytes of the sweep kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "k_sweep_c2.md")
    try:
        for line in open(path):
            if line.startswith("traffic_per_launch_bytes:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


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


def _output_fault_sample(flst_text, n):
    """First n output faults (pin 0) of an @pins list, as plain .flst text."""
    toks = flst_text.split()
    pins = toks[0] == "@pins"
    if pins:
        toks = toks[1:]
    F = int(toks[0])
    out = []
    step = 3 if pins else 2
    for i in range(F):
        site, val = toks[1 + step * i], toks[2 + step * i]
        pin = toks[3 + step * i] if pins else "0"
        if pin == "0":
            out.append("%s %s" % (site, val))
            if len(out) == n:
                break
    return "%d\n%s\n" % (len(out), "\n".join(out))


def cpu_baseline(w, target_s=15.0):
    """The reference simulator (else the CPU port) on a bounded sample of the
    workload: S output faults x R rounds, all faults sharded over threads."""
    from tests.oracle_lib import Oracle, Reference, ref_available
    threads = max(1, min(64, os.cpu_count() or 1))
    full = Oracle(w["ckt"], "0\n", w["ptn"])
    if ref_available():
        kind = "reference"
        fl = _output_fault_sample(w["flst"], 4 * threads)
        ref = Reference(w["ckt"], fl, words=full.words, P=full.P, n_pi=full.n_pi)
        ref.simulate(rd0=0, rd1=1, threads=threads)          # load workers, calibrate
        per_round = max(ref.seconds, 1e-3)
        R = int(max(1, min(full.W, target_s / per_round)))
        ref.simulate(rd0=0, rd1=R, threads=threads)
        secs, nf = ref.seconds, ref.F
    else:
        kind = "port"
        fl = _output_fault_sample(w["flst"], 32 * threads)
        o = Oracle(w["ckt"], fl, w["ptn"])
        t0 = time.perf_counter()
        o.simulate(rd0=0, rd1=1, mode=0, threads=threads)
        per_round = max(time.perf_counter() - t0, 1e-3)
        R = int(max(1, min(full.W, target_s / per_round)))
        t0 = time.perf_counter()
        o.simulate(rd0=0, rd1=R, mode=0, threads=threads)
        secs, nf = time.perf_counter() - t0, len(o.faults)
    value = nf * R * 64 / secs
    return {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": "%d output faults x %d rounds (%d patterns) of the %s workload, %.1f s"
                      % (nf, R, R * 64, WORKLOAD, secs)}


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return
    from lsim_b200 import gen
    w = gen.workload(WORKLOAD)
    n_faults = int(w["flst"].split()[1 if w["flst"].startswith("@pins") else 0])
    for _ in range(args.warmup):
        cpu_baseline(w, target_s=2.0)
    vals, secs = [], []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        b = cpu_baseline(w, target_s=args.ref_seconds)
        vals.append(b["value"])
    elapsed = time.perf_counter() - t0
    value = statistics.median(vals)
    P = 65536
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * n_faults * P / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": _workload_desc(n_faults), "mode": "count",
                       "timed": "bounded sample per step; ms_per_step extrapolated to the full job"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": b["cores"], "kind": b["kind"],
                             "sample": b["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": elapsed}
    print(json.dumps(line), flush=True)


def _workload_desc(n_faults):
    return ("c2: 200,000 gates, 1,000 PI, 1,000 PO, 150 levels, mean fan-in 2.2; %d collapsed "
            "output+input-pin SA faults; 65,536 patterns" % n_faults)


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
        if faults_sharded:
            return shard.merge_fault_shards(res, my_faults, F_all, info.num_rounds, device="cuda")
        return shard.merge_results(res, rank * P, rank == world - 1, world * info.num_rounds,
                                   device="cuda")

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
    sweep_ms, sweep_bytes, tiles, launches = 0.0, 0, 0, 0
    for _ in range(args.steps):
        sim.run(stream=sp, tune=True)
        merged = merge(sim.results())
        st = sim.stats()
        sweep_ms += st["ms_sweep"]
        sweep_bytes += st["sweep_alg_bytes"]
        tiles += st["n_tiles"]
        launches += st["kernel_launches"]
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
    peak, peak_src = _peaks()
    per_launch_bytes = sweep_bytes / max(1, tiles)
    per_launch_s = sweep_ms / max(1, tiles) / 1e3
    achieved = per_launch_bytes / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
    st = sim.stats()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if faults_sharded else "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic",
        "config": {"workload": _workload_desc(F_all), "faults": F_all, "patterns": P,
                   "elements": info.num_elements, "mode": "count",
                   "parallelism": ("1 GPU" if world == 1 else
                                   "%s-sharded x%d" % ("fault" if faults_sharded else "pattern", world)),
                   "l2": "inputs larger than L2: good-machine words %.2f GB rewritten each step"
                         % (info.num_elements * info.num_rounds * 8 / 1e9),
                   "sweep": {"words_per_item": st["words_per_item"],
                             "block_threads": st["block_threads"], "blocks": st["blocks"],
                             "ctas_per_sm": st["ctas_per_sm"], "smem_bytes": st["smem_bytes"],
                             "max_live": st["max_live"],
                             "shape": "autotuned during warm-up on a strided sample of the "
                                      "first tile's sweeps", "tune_ms": tune_ms}},
        "e2e": {"value": e2e, "unit": UNIT,
                "h2d_bytes_per_step": int(words.nbytes),
                "d2h_bytes_per_step": int(F * 17)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": _profile_traffic(),
                     "kernel": "k_sweep", "peak_source": peak_src + " (MEASURED_PEAKS.json hbm_gbs)",
                     "per_launch_alg_bytes": per_launch_bytes, "per_launch_ms": per_launch_s * 1e3},
        "breakdown_ms_per_step": {"good": st["ms_good"], "sweep": st["ms_sweep"],
                                  "ffr": st["ms_ffr"], "compute": st["ms_compute"],
                                  "total": st["ms_total"]},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w, target_s=args.ref_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_batch(args):
    """Batched configuration: one batch of 256 circuits against 256 plain runs."""
    import torch
    from lsim_b200 import Batch, Simulator, gen
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    cfgs = gen.batch_configs(args.circuits, seed=0)
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
    for _ in range(max(0, args.warmup - 1)):
        b.run(tune=True, stream=sp)
    for p in plains:
        p.run(stream=sp, tune=True)
    clocks = ClockSampler(0)
    clocks.start()
    ms_batch = timed(lambda: b.run(tune=True, stream=sp), args.steps)
    st = b.stats()
    ms_serial = timed(lambda: b.run(tune=True, concurrent=False, stream=sp), args.steps)
    ms_plain = timed(lambda: [p.run(stream=sp, tune=True) for p in plains], args.steps)
    clk = clocks.stop()
    plain_launches = sum(p.stats()["kernel_launches"] for p in plains)
    # e2e: every input from host memory each step
    ms_batch_e2e = timed(lambda: b.run(tune=True, reupload=True, stream=sp), args.steps)
    st_e2e = b.stats()
    words = [p.patterns() for p in plains]
    pinned = [torch.from_numpy(wd.ravel()).pin_memory().numpy() for wd in words]

    def plain_e2e():
        for p, wd, m in zip(plains, pinned, members):
            p.set_patterns(wd, m.info().num_patterns)
            p.run(stream=sp, tune=True)
            p.results()
    ms_plain_e2e = timed(plain_e2e, args.steps)
    # phase split of one step of each arm (batch without the graph)
    b.run(tune=True, graph=False, stream=sp)
    st_ng = b.stats()
    classes = b.classes()
    phases = {"batch": {k: st_ng[k] for k in ("ms_good", "ms_sweep", "ms_ffr", "ms_total")},
              "plain": {k: sum(p.stats()[k] for p in plains)
                        for k in ("ms_good", "ms_sweep", "ms_ffr", "ms_total")}}
    # results agree with the plain path on every circuit
    same = all(np.array_equal(m.results(), p.results()) for m, p in zip(members, plains))
    peak, peak_src = _peaks()
    sweep_s = st["ms_compute"] / 1e3
    line = {
        "metric": "fault×pattern evals/s (batched, %d circuits)" % args.circuits,
        "value": FP * args.steps / (ms_batch / 1e3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_batch / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic",
        "config": {"workload": "c4: %d circuits, %d-%d gates (median %d), 10-120 levels, SA0/SA1 "
                               "on every gate output (%d faults), 1,024-16,384 patterns"
                               % (args.circuits, min(gates), max(gates), int(np.median(gates)), F),
                   "fault_patterns_per_step": FP, "mode": "count",
                   "sweep": {k: st[k] for k in ("words_per_item", "block_threads", "ctas_per_sm",
                                                "blocks", "smem_bytes", "n_classes")},
                   "graph": bool(st["graph_used"]), "tune_ms": tune_ms,
                   "first_run_s": first_s, "generate_s": gen_s},
        "plain_sequential": {"value": FP * args.steps / (ms_plain / 1e3),
                             "ms_per_step": ms_plain / args.steps,
                             "gpu_launches_per_step": int(plain_launches)},
        "batch_over_plain": ms_plain / ms_batch,
        "batch_serial_classes": {"value": FP * args.steps / (ms_serial / 1e3),
                                 "ms_per_step": ms_serial / args.steps},
        "e2e": {"value": FP * args.steps / (ms_batch_e2e / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": int(st_e2e["h2d_bytes"]),
                "d2h_bytes_per_step": int(st_e2e["d2h_bytes"])},
        "plain_sequential_e2e": {"value": FP * args.steps / (ms_plain_e2e / 1e3),
                                 "ms_per_step": ms_plain_e2e / args.steps},
        "gpu_launches": int(st["kernel_launches"]) * args.steps,
        "breakdown_ms_per_step": {"compute": st["ms_compute"], "d2h": st["ms_d2h"],
                                  "total": st["ms_total"]},
        "roofline": {"bound": "hbm", "achieved": st["sweep_alg_bytes"] / sweep_s / 1e9,
                     "peak": peak, "unit": "GB/s",
                     "frac": st["sweep_alg_bytes"] / sweep_s / 1e9 / peak, "traffic": None,
                     "kernel": "whole batch (good + sweeps + tracing)",
                     "peak_source": peak_src + " (MEASURED_PEAKS.json hbm_gbs)"},
        "phases_ms_per_step": phases,
        "classes": classes,
        "results_equal_plain": same,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    b.close()


def run_serve(args):
    """Serving configuration: requests against 32 resident circuits, served
    by the server (waves on concurrent slots) and by the plain path one job
    at a time, at a burst and at Poisson arrival rates."""
    import threading
    import torch
    from lsim_b200 import Server, Simulator, gen
    torch.cuda.set_device(0)
    rng = np.random.default_rng(0)
    cfgs = gen.serve_configs(args.circuits if args.circuits != 256 else 32, seed=0)
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
    n_req = args.requests
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

    srv = Server(0, slots=args.slots, slot_bytes=args.slot_gib << 30)
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
    for f in args.rates:
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
                   "fault_patterns": FP, "slots": args.slots, "slot_gib": args.slot_gib,
                   "generate_s": gen_s, "add_circuits_s": add_s,
                   "resident_bytes": st["resident_bytes"], "slot_bytes": st["slot_bytes"],
                   "rates": "fractions of the plain path's burst capacity (%.2f requests/s)" % cap},
        "burst": {"server": burst_srv, "plain": burst_plain},
        "poisson": rows,
        "results_equal_plain": same,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    srv.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default=WORKLOAD, help="c2 (default) or another gen.WORKLOADS key")
    ap.add_argument("--shard", default="patterns", choices=["patterns", "faults"],
                    help="with --gpus N > 1: each rank its own pattern block (weak scaling, "
                         "default) or its part of the fault list (strong scaling)")
    ap.add_argument("--circuits", type=int, default=256,
                    help="circuits for --workload c4 (default 256) or c5 (default 32)")
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
        w = gen.workload(args.workload)
        sim = Simulator(0)
        sim.read_text(w["ckt"], w["flst"], w["ptn"])
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
                          "patterns": info.num_patterns, "elements": info.num_elements,
                          "mode": "drop" if args.drop else "count", "wall_s": wall,
                          "detected": int(res["detected"].sum()), "stats": st}))
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
