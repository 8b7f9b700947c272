"""Benchmark: batched RC-net timing (BFS flattening + Elmore, 4 corners) on
1M synthetic nets, plus levelization of a 5M-pin timing graph.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one fused pass of otg_rc_timing over the whole batch (1M nets,
log-uniform 2..4096 nodes, ~5.4e8 nodes, generated on the device).  Inputs
(~15 GB) and outputs (~45 GB) are far larger than the 126 MB L2, so no
flush is needed between steps.  Prints ONE JSON line (rank 0).

--impl reference times the reference's own CPU path (Rct::update_rc_timing
in a Cpp-Taskflow parallel_for over all host threads, oracle/_ref) on a
bounded sample of the same workload, in the same metric.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RC-tree nodes/s (Elmore, 4 corners) & levelize edges/s; incr. p50/p99 latency"
NUM_NETS = 1_000_000
SEED = 2024
LV_PINS, LV_EDGES, LV_LEVELS = 5_000_000, 12_000_000, 200
TUNE_NETS = 50_000
SPEF_NETS = 20_000
# DRAM bytes per node of one RC pass (dram__bytes_read.sum + dram__bytes_write.sum
# over the 8 launches of one pass), from an ncu capture of 30k nets of the same
# net-size distribution with the autotuned table: 2.204 GB / 15,951,150 nodes
# (profiles/rc_pass_dram_traffic_30k_nets.md).  The pass's traffic grows with
# its nodes, so a step's traffic is this times the step's nodes.  (At 30k nets
# part of the small classes' writes is still in L2 when the capture ends; the
# dominant kernel alone moves 152.8 B/node.)
RC_DRAM_BYTES_PER_NODE = 138.2
FU_GATES = 50_000
FU_REPS = 5
FU_CHANGE = 0.01  # fraction of the nets a change SPEF re-draws
# incremental sizing loop
INC_GATES, INC_ITERS, INC_FRAC, INC_PLAIN_ITERS, INC_REF_ITERS = 200_000, 1000, 0.005, 100, 3
# serving
SRV_DESIGNS, SRV_PINS_LO, SRV_PINS_HI = 16, 10_000, 2_000_000
# offered rates: below both paths' capacity, between the plain path's (about
# 180 req/s on the 16 designs) and the batched one's (about 450), and above both
SRV_RATES, SRV_MAX_REQ, SRV_SAT_REQ, SRV_REF_REQ = (100, 300, 1_000), 2_000, 3_000, 12
SRV_PINS_PER_GATE = 2.75  # designgen: pins per gate of a design


def algorithmic_bytes(num_nets, total_nodes, num_sinks):
    """Bytes a perfect fused pass must move: read edges 8 + res 4 + cap 16 per
    node (edges/res per non-root node), write edges 8 + node2bfs 4 + pid 4 +
    load/delay/ldelay/impulse 64; per net nodes_start 4 + roots 4 +
    sinks_start 4 + driver slew 16; per sink its id 4 + slew 16."""
    E = total_nodes - num_nets
    return (E * (8 + 4 + 8) + total_nodes * (16 + 4 + 4 + 64) + num_nets * (4 + 4 + 4 + 16)
            + num_sinks * (4 + 16))


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": mx or None, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if args.impl == "ours":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    elif args.impl == "ours":
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, x):
    """The maximum of x over all ranks (a device tensor under NCCL, a host
    one under gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_nets(rank, nets, lo, hi):
    """This rank's share of a weak-scaling run: its own seeded nets (the
    same count and size distribution on every rank, no data exchanged)."""
    from opentimer_b200 import workloads
    return workloads.net_sizes(SEED + rank, nets, lo, hi)


def load_workloads():
    """opentimer_b200/workloads.py as a standalone module (numpy only), so
    the reference arm sizes the workload without loading the package and
    its library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "otg_workloads", os.path.join(ROOT, "opentimer_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def headline_config(nets, total_nodes, lo, hi, world):
    """The `config` of the headline line, the same dict in both arms."""
    return {"workload": f"batched Elmore: {nets} RC nets/GPU, log-uniform {lo}..{hi} nodes, "
                        "70% random recursive trees / 30% chains, 4 corners, sink slews",
            "num_nets_per_gpu": nets, "total_nodes_per_gpu": total_nodes, "seed": SEED,
            "l2": "inputs and outputs (>60 GB) far exceed L2; no flush needed",
            "parallelism": f"replicas x{world} (nets shard with no collective)"}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ------------------------------------------------------------ CPU baseline

def cpu_sample(ns_full, g, sample_nets):
    """Host copy of the first `sample_nets` nets of the device workload."""
    import oracle as O
    ns = ns_full[:sample_nets + 1].copy()
    V = int(ns[-1])
    E = V - sample_nets
    f = O.Forest(ns, g["edges"][:E].cpu().numpy(), g["roots"][:sample_nets].cpu().numpy(),
                 g["res"][:E].cpu().numpy(), g["cap"][:V].cpu().numpy())
    return f


def time_reference_cpu(f, threads):
    """Reference Rct::update_rc_timing over the sample with `threads` host
    threads (reference build when present, else the oracle port on 1 core)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if O.ref_available():
        t0 = time.perf_counter()
        st, _ = O.ref_rct_update(f, threads, readback=True)
        dt = time.perf_counter() - t0
        if st != 0:
            raise RuntimeError("reference CPU path failed")
        return dt, "reference", threads
    t0 = time.perf_counter()
    st, _ = O.elmore_cpu_f32(f)
    return time.perf_counter() - t0, "port", 1


def sample_nets_for_budget(ns, seconds, est_nodes_per_s):
    """Largest net prefix whose node count fits `seconds` of CPU work."""
    target = seconds * est_nodes_per_s
    k = int(np.searchsorted(ns, target))
    return max(1000, min(len(ns) - 1, k))


def calibrate_cpu(make_forest, ns, threads):
    """Nodes/s of the CPU path on a 2000-net prefix (to size the sample)."""
    f = make_forest(2000)
    dt, _, _ = time_reference_cpu(f, threads)
    return f.total_nodes / max(dt, 1e-6)


# ------------------------------------------------------------------ main

def run_reference(args, world, rank):
    """--impl reference: the reference's own CPU path (Rct::update_rc_timing
    in a Cpp-Taskflow parallel_for over all host threads, oracle/_ref) on
    the headline workload, rank 0 only.  Each timed step takes its own
    1/steps of the workload's nets, so the timed steps together cover all
    of its nets once; warm-up steps repeat the first slices.  Inputs come
    from the oracle's host generator (bit-identical to the device
    generator), built outside the timed region; the product library is not
    loaded in this arm."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    wl = load_workloads()
    ns_full = wl.net_sizes(SEED, args.nets, args.min_nodes, args.max_nodes).astype(np.int64)
    N, V_full = args.nets, int(ns_full[-1])
    threads = os.cpu_count() or 1
    steps = max(1, args.steps)
    cuts = [int(round(N * k / steps)) for k in range(steps + 1)]
    kind = "reference" if O.ref_available() else "port"
    times, nodes = [], 0
    for i in range(args.warmup + args.steps):
        k = (i - args.warmup) % steps if i >= args.warmup else i % steps
        a, b = cuts[k], cuts[k + 1]
        f, _, _ = O.synth_forest(SEED, ns_full[a:b + 1], first_net=a, threads=threads)
        if kind == "reference":
            t0 = time.perf_counter()
            st, _ = O.ref_rct_update(f, threads, readback=False)
            dt = time.perf_counter() - t0
            if st != 0:
                raise RuntimeError("reference CPU path failed")
        else:
            t0 = time.perf_counter()
            O.elmore_cpu_f32(f)
            dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            nodes += f.total_nodes
        del f
    total = sum(times)
    value = nodes / total
    cores = threads if kind == "reference" else 1
    line = {
        "metric": METRIC, "value": value, "unit": "nodes/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; the GPU arm's generator restated on the host)",
        "config": headline_config(N, V_full, args.min_nodes, args.max_nodes, world),
        "cpu_baseline": {"value": value, "unit": "nodes/s", "cores": cores, "kind": kind,
                         "sample": f"each timed step one 1/{steps} slice of the {N} nets; the "
                                   f"{args.steps} timed steps cover {nodes} of {V_full} nodes; "
                                   "Rct built and timed per net as Net::_update_rc_timing "
                                   "does, results left in the Rct nodes"},
        "e2e": {"value": value, "unit": "nodes/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def autotune_on(seed, nets, lo, hi, dev):
    """Runs the RC-pass autotuner on a seeded sample with the workload's
    net-size distribution (a different seed from the timed forest) and
    leaves its tuning applied.  Returns (tuning, seconds)."""
    import torch
    import opentimer_b200 as otg
    from opentimer_b200 import workloads
    t0 = time.perf_counter()
    ns = torch.from_numpy(workloads.net_sizes(seed, nets, lo, hi)).to(dev)
    g = otg.synth_forest(seed, ns)
    b = otg.RcBatch(ns, g["edges"], g["roots"], g["res"], g["cap"], sinks_start=g["sinks_start"],
                    sink_nodes=g["sink_nodes"], driver_slew=g["driver_slew"], max_net_nodes=hi)
    t = otg.autotune(b)
    del b, g, ns
    torch.cuda.empty_cache()
    return t, time.perf_counter() - t0


def run_ours(args, world, rank, local):
    import torch
    import opentimer_b200 as otg
    from opentimer_b200 import workloads
    dev = torch.device("cuda", local if world > 1 else 0)
    stream = torch.cuda.current_stream(dev)

    # ---- workload (per rank: its own 1M nets -> weak scaling)
    tuning, tune_s = None, 0.0
    if args.tuning:  # a saved tuning (a profiler run replays the timed run's choice)
        src = args.tuning
        tuning = json.load(open(src)) if os.path.exists(src) else json.loads(src)
        otg.set_tuning(tuning)
    elif not args.no_autotune:
        tuning, tune_s = autotune_on(SEED + 100 + rank, min(TUNE_NETS, args.nets), args.min_nodes,
                                     args.max_nodes, dev)
    ns_np = rank_nets(rank, args.nets, args.min_nodes, args.max_nodes)
    ns = torch.from_numpy(ns_np).to(dev)
    g = otg.synth_forest(SEED + rank, ns)
    torch.cuda.synchronize()
    N, V = args.nets, int(ns_np[-1])
    S = int(g["sink_nodes"].numel())
    batch = otg.RcBatch(ns, g["edges"], g["roots"], g["res"], g["cap"],
                        sinks_start=g["sinks_start"], sink_nodes=g["sink_nodes"],
                        driver_slew=g["driver_slew"], max_net_nodes=args.max_nodes)
    for _ in range(args.warmup):
        batch.run(stream)
    batch.check(stream)
    torch.cuda.synchronize()
    barrier(world)
    l0 = otg.kernel_launches()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        torch.cuda.synchronize()
        barrier(world)
        ev0.record(stream)
        for _ in range(args.steps):
            batch.run(stream)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    launches = otg.kernel_launches() - l0
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(world, ms)
    batch.check(stream)
    # the timed run's own outputs, checked on a sample of its nets
    parity = _section(check_headline_outputs, batch, ns_np, SEED + rank) \
        if not args.no_parity else None
    value = world * V / (ms / 1e3)
    peak, peak_kind = load_peaks()
    abytes = algorithmic_bytes(N, V, S)
    achieved = abytes / (ms / 1e3) / 1e9

    # ---- end to end through the host C ABI (pinned host buffers)
    e2e = None
    SECTION_WALL_S["headline"] = round(time.perf_counter() - T_START, 2)
    t0 = time.perf_counter()
    if not args.no_e2e:
        e2e = run_e2e(args, world, g, ns_np, N, V, S, dev, batch)
    SECTION_WALL_S["run_e2e"] = round(time.perf_counter() - t0, 2)

    # ---- levelization (5M pins, 12M edges, 200 levels)
    t0 = time.perf_counter()
    lv = run_levelize(args, world, dev) if not args.no_levelize else None
    SECTION_WALL_S["run_levelize"] = round(time.perf_counter() - t0, 2)

    line = {
        "metric": METRIC, "value": value, "unit": "nodes/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded, generated on the device)",
        "config": headline_config(N, V, args.min_nodes, args.max_nodes, world),
        "sinks_per_gpu": S,
        "tuning": tuning or "default",
        "autotune": ("given (--tuning)" if args.tuning else
                     f"otg_rc_autotune on {min(TUNE_NETS, args.nets)} nets of the same "
                     f"distribution (another seed), {tune_s:.1f} s, before warm-up")
        if tuning else "off",
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": RC_DRAM_BYTES_PER_NODE * V,
                     "traffic_source": "ncu dram bytes per node of one pass (30k-net capture) "
                                       "x this step's nodes",
                     "kernel": "otg_rc_timing fused pass (classify + size-class launches)",
                     "algorithmic_bytes_per_step": abytes, "peak_kind": peak_kind},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if e2e:
        line["e2e"] = e2e
    if parity is not None:
        line["parity"] = parity
    if lv:
        line["levelize"] = lv
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = _section(cpu_baseline, g, ns_np)
        # the free memory of the timed batch is not needed by the reference run
        line["reference_gpu_rc"] = _section(reference_gpu_rc, ns_np, SEED + rank)
    # the per-GPU incremental and serving loops (one GPU only)
    if world == 1 and not (args.no_incremental and args.no_serving):
        del batch, g
        torch.cuda.empty_cache()
    if world == 1 and not args.no_incremental:
        line["incremental"] = _section(run_incremental,
                                       baseline=line.get("cpu_baseline") if rank == 0 else None)
    if world == 1 and not args.no_serving:
        line["serving"] = _section(run_serving,
                                   baseline=line.get("cpu_baseline") if rank == 0 else None)
    # reference runs of the other sections belong to the CPU-baseline leg
    base = line.get("cpu_baseline")
    if base is not None and lv:
        base["levelize"] = _section(levelize_baseline, lv)
        if parity is not None and isinstance(base["levelize"], dict):
            for k in ("levels_match_reference", "levels_match_port"):
                if k in base["levelize"]:
                    parity[k] = base["levelize"][k]
    if rank == 0 and not args.no_spef:
        line["spef_ingest"] = _section(run_spef, base)
    if world == 1 and not args.no_full_update:
        line["full_update"] = _section(run_full_update, baseline=base if rank == 0 else None)
    if world == 1 and not args.no_huge:
        line["huge_nets"] = _section(run_huge)
    line["section_wall_s"] = dict(SECTION_WALL_S, total=round(time.perf_counter() - T_START, 1))
    return line


PARITY_BINS = (2, 33, 129, 257, 513, 1025, 2049, 4097)  # warp path, then block classes
PARITY_NETS_PER_BIN = 300


def _net_max(ns, x):
    sizes = np.diff(ns)
    m = np.maximum.reduceat(np.abs(x), ns[:-1], axis=0)
    return np.repeat(m, sizes, axis=0)


def check_headline_outputs(batch, ns_np, seed):
    """The timed run's outputs on a seeded sample of its nets: PARITY_NETS_PER_BIN
    nets from each size bin (every size class of the pass), inputs rebuilt
    on the host by the oracle's generator (bit-identical to the device
    generator), outputs gathered from the device batch.  BFS slots, pid and
    directed edges against the oracle's BFS rule (bit-exact); load, delay,
    ldelay and impulse against the reference's own CPU Rct (oracle/_ref,
    else the oracle's bit-exact restatement of it) within |d| <= 1e-5|ref| +
    1e-6 max_net|ref|; sink slews within that tolerance carried through
    sqrt; and the largest error against an FP64 evaluation, for ours and for
    the reference, per quantity (max |x - exact| / max_net|exact|)."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ns64 = ns_np.astype(np.int64)
    sizes = np.diff(ns64)
    rng = np.random.default_rng(seed + 99)
    pick = []
    for lo, hi in zip(PARITY_BINS[:-1], PARITY_BINS[1:]):
        idx = np.nonzero((sizes >= lo) & (sizes < hi))[0]
        if len(idx):
            pick.append(rng.choice(idx, min(PARITY_NETS_PER_BIN, len(idx)), replace=False))
    nets = np.sort(np.concatenate(pick + [np.argsort(sizes)[-8:]]))
    nets = np.unique(nets)
    # host inputs of the sampled nets, one net at a time from the generator
    parts = [O.synth_forest(seed, ns64[i:i + 2], first_net=int(i), threads=1) for i in nets]
    n = sizes[nets]
    fs_ns = np.zeros(len(nets) + 1, np.int64)
    fs_ns[1:] = np.cumsum(n)
    f = O.Forest(fs_ns, np.concatenate([p[0].edges for p in parts]),
                 np.concatenate([p[0].roots for p in parts]),
                 np.concatenate([p[0].res for p in parts]),
                 np.concatenate([p[0].cap for p in parts]))
    slew = np.concatenate([p[1] for p in parts])
    # device outputs of those nets
    dev = batch.node2bfs.device
    node_idx = np.concatenate([np.arange(ns64[i], ns64[i + 1]) for i in nets])
    edge_idx = np.concatenate([np.arange(ns64[i] - i, ns64[i + 1] - i - 1) for i in nets])
    ti = torch.from_numpy(node_idx).to(dev)
    te = torch.from_numpy(edge_idx).to(dev)
    got = {k: getattr(batch, k).index_select(0, ti).cpu().numpy()
           for k in ("node2bfs", "pid", "load", "delay", "ldelay", "impulse")}
    got["edges"] = batch.edges.index_select(0, te).cpu().numpy()
    ss_dev = batch.sinks_start.cpu().numpy().astype(np.int64)
    sink_idx = np.concatenate([np.arange(ss_dev[i], ss_dev[i + 1]) for i in nets])
    ts = torch.from_numpy(sink_idx).to(dev)
    got_sn = batch.sink_nodes.index_select(0, ts).cpu().numpy()
    got_ss = batch.sink_slew.index_select(0, ts).cpu().numpy()
    sn_count = ss_dev[nets + 1] - ss_dev[nets]
    f_ss = np.zeros(len(nets) + 1, np.int64)
    f_ss[1:] = np.cumsum(sn_count)
    out = {"nets_checked": int(len(nets)), "nodes_checked": int(f.total_nodes),
           "sinks_checked": int(len(sink_idx)),
           "sample": f"{PARITY_NETS_PER_BIN} seeded nets per size bin {list(PARITY_BINS)} "
                     "plus the 8 largest, from the timed batch after the timed steps"}
    st, e, n2b, pid, _ = O.bfs(f)
    out["bfs_pid_edges_bit_exact"] = bool(
        st == 0 and np.array_equal(got["node2bfs"], n2b) and np.array_equal(got["pid"], pid)
        and np.array_equal(got["edges"], e))
    base = np.repeat(fs_ns[:-1], n)
    local = {q: got[q][base + got["node2bfs"]] for q in ("load", "delay", "ldelay", "impulse")}
    threads = os.cpu_count() or 1
    if O.ref_available():
        st, ref = O.ref_rct_update(f, threads, readback=True)
        out["reference"] = "the reference's Rct::update_rc_timing (oracle/_ref)"
    else:
        st, ref = O.elmore_cpu_f32(f)
        out["reference"] = "the oracle's restatement of Rct::update_rc_timing"
    st64, ex = O.elmore_f64(f)
    errs, rel_ours, rel_ref = {}, {}, {}
    for q, r, x in zip(("load", "delay", "ldelay", "impulse"), ref, ex):
        g = local[q].astype(np.float64)
        tol = np.maximum(1e-5 * np.abs(r) + 1e-6 * _net_max(fs_ns, r), np.finfo(np.float32).tiny)
        errs[q] = float(np.max(np.abs(g - r) / tol))
        nm = np.maximum(_net_max(fs_ns, x), 1e-30)
        rel_ours[q] = float(np.max(np.abs(g - x) / nm))
        rel_ref[q] = float(np.max(np.abs(r.astype(np.float64) - x) / nm))
    out["max_err_over_tol"] = errs
    out["tolerance"] = "|ours - ref| <= 1e-5 |ref| + 1e-6 max_net|ref| per node, corner, quantity"
    out["max_rel_vs_fp64"] = rel_ours
    out["reference_max_rel_vs_fp64"] = rel_ref
    # sink slews from the reference impulse
    want = O.sink_slew(f, f_ss.astype(np.int32), got_sn, slew, ref[3])
    nb = np.repeat(fs_ns[:-1], sn_count)
    imp = ref[3][nb + got_sn]
    imp_max = _net_max(fs_ns, ref[3])[nb + got_sn]
    tol = (1e-5 * np.abs(imp) + 1e-6 * imp_max) / (2 * np.abs(want)) + 1e-6 * np.abs(want)
    out["sink_slew_max_err_over_tol"] = float(np.max(np.abs(got_ss - want) / tol)) \
        if len(want) else 0.0
    out["pass"] = bool(out["bfs_pid_edges_bit_exact"] and st == 0 and st64 == 0 and
                       max(errs.values()) <= 1.0 and out["sink_slew_max_err_over_tol"] <= 1.0)
    return out


SECTION_WALL_S = {}  # host wall seconds of every section, for the line


def _section(fn, *args, **kw):
    """Runs a section after the headline measurement: a failure is reported
    in the line ({"error": ...}, traceback on stderr) instead of losing the
    headline numbers.  Its wall time goes to SECTION_WALL_S."""
    t0 = time.perf_counter()
    try:
        return fn(*args, **kw)
    except Exception as e:  # noqa: BLE001 -- reported, not swallowed
        import traceback
        traceback.print_exc()
        return {"error": f"{type(e).__name__}: {e}"}
    finally:
        name = fn.__name__
        SECTION_WALL_S[name] = round(SECTION_WALL_S.get(name, 0.0) + time.perf_counter() - t0, 2)


def run_e2e(args, world, g, ns_np, N, V, S, dev, batch):
    """Same pass through otg_rc_timing_host: pinned host inputs -> device ->
    compute -> host outputs, all inside the timed region, `steps` times.
    Afterwards the host outputs of the first and last 20k nets are compared
    with the device-resident pass's (`batch`, the same inputs): identical
    bits expected."""
    import torch
    import opentimer_b200 as otg
    def pin(t):
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t)
        return h
    h_ns = torch.from_numpy(ns_np).pin_memory()
    h_edges = pin(g["edges"])
    h_roots, h_res, h_cap = pin(g["roots"]), pin(g["res"]), pin(g["cap"])
    h_ss, h_sn, h_slew = pin(g["sinks_start"]), pin(g["sink_nodes"]), pin(g["driver_slew"])
    outs = {k: torch.empty(V, dtype=torch.int32).pin_memory() for k in ["node2bfs", "pid"]}
    for k in ["load", "delay", "ldelay", "impulse"]:
        outs[k] = torch.empty(V, 4, dtype=torch.float32).pin_memory()
    sink_slew = torch.empty(S, 4, dtype=torch.float32).pin_memory()
    P = lambda t: t.data_ptr()  # noqa: E731
    f = otg.RcForest(N, V, P(h_ns), P(h_edges), P(h_roots), P(h_res), P(h_cap),
                     P(outs["node2bfs"]), P(outs["pid"]), P(outs["load"]), P(outs["delay"]),
                     P(outs["ldelay"]), P(outs["impulse"]), P(h_ss), P(h_sn), P(h_slew),
                     P(sink_slew))
    L = otg.lib()
    for _ in range(1):
        otg.check("otg_rc_timing_host", L.otg_rc_timing_host(ctypes.byref(f)))
    steps = max(1, args.steps)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(steps):
        otg.check("otg_rc_timing_host", L.otg_rc_timing_host(ctypes.byref(f)))
    dt = (time.perf_counter() - t0) / steps
    dt = max_over_ranks(world, dt)
    E = V - N
    h2d = 4 * (N + 1) + 8 * E + 4 * N + 4 * E + 16 * V + 4 * (N + 1) + 4 * S + 16 * N
    d2h = 8 * E + 4 * V + 4 * V + 64 * V + 16 * S
    # the copies carried the pass's results: the first and last 20k nets
    # against the device-resident pass on the same inputs, bit for bit
    ok = True
    for a, b in ((0, min(N, 20_000)), (max(0, N - 20_000), N)):
        v0, v1 = int(ns_np[a]), int(ns_np[b])
        for k in ["node2bfs", "pid", "load", "delay", "ldelay", "impulse"]:
            hd = outs[k][v0:v1].numpy()
            dd = getattr(batch, k)[v0:v1].cpu().numpy()
            ok = ok and np.array_equal(hd.view(np.int32), dd.view(np.int32))
        s0, s1 = int(h_ss[a]), int(h_ss[b])
        ok = ok and np.array_equal(sink_slew[s0:s1].numpy().view(np.int32),
                                   batch.sink_slew[s0:s1].cpu().numpy().view(np.int32))
    return {"value": world * V / dt, "unit": "nodes/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": dt * 1e3, "steps": steps,
            "host_buffers": "pinned (torch.pin_memory)",
            "outputs_match_device_pass": bool(ok),
            "path": "otg_rc_timing_host (chunked H2D / compute / D2H on two streams)"}


def run_levelize(args, world, dev):
    import torch
    import opentimer_b200 as otg
    from opentimer_b200 import workloads
    fs, fi, od, f0 = workloads.pin_dag(SEED, LV_PINS, LV_EDGES, LV_LEVELS)
    t = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
    lb = otg.LevelizeBatch(t(fs), t(fi), t(od), t(f0))
    stream = torch.cuda.current_stream(dev)
    for _ in range(3):
        lb.run(stream)
    lb.check(stream)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    steps = 10
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        lb.run(stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    ms = max_over_ranks(world, ms)
    lb.check(stream)
    L, emitted = [int(x) for x in lb.counts.tolist()]
    n, E = len(od), len(fi)
    lv_bytes = 12 * E + 16 * n
    # the same through host arrays (otg_levelize_host: copies in, levelize,
    # copies out), as a Timer hands its CSR over
    otg.levelize_host(fs, fi, od, f0)
    t0 = time.perf_counter()
    otg.levelize_host(fs, fi, od, f0)
    host_ms = 1e3 * (time.perf_counter() - t0)
    return {"edges_per_s": world * E / (ms / 1e3), "ms": ms, "pins": n, "edges": E,
            "levels": L, "emitted": emitted, "us_per_level": 1e3 * ms / max(L, 1),
            "host_path_ms": host_ms,
            "hbm_gbs": lv_bytes / (ms / 1e3) / 1e9,
            "workload": f"pin DAG {n} pins, {E} edges, {L} levels (seeded)"}


def levelize_baseline(ours):
    """The levelization workload (the same seeded pin DAG) through the
    reference's own toposort_compute_cuda loop (oracle/_ref: its
    toposort_advance kernel, one launch and one blocking copy per level,
    with its allocations and copies, as the Timer calls it) and through the
    oracle's restatement of the frontier Kahn on one host core.  Both are
    checked against our levels."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from opentimer_b200 import workloads
    fs, fi, od, f0 = workloads.pin_dag(SEED, LV_PINS, LV_EDGES, LV_LEVELS)
    n = len(od)
    out = {"unit": "ms per levelization", "kind": "reference",
           "ours_device_ms": ours["ms"]}
    t0 = time.perf_counter()
    order, ends, _ = O.levelize(n, fs, fi, od, f0)
    out["port_cpu_ms"] = 1e3 * (time.perf_counter() - t0)
    out["port_cpu_cores"] = 1
    out["levels_match_port"] = bool(len(ends) - 1 == ours["levels"])
    if O.ref_available():
        O.ref_toposort_gpu(n, fs, fi, od, f0)  # warm-up (context, module load)
        t0 = time.perf_counter()
        fr, rends = O.ref_toposort_gpu(n, fs, fi, od, f0)
        out["value"] = 1e3 * (time.perf_counter() - t0)
        out["what"] = ("the reference's toposort_compute_cuda loop on the B200 (oracle/_ref), "
                       "host arrays in and out, as the Timer calls it")
        out["levels_match_reference"] = bool(
            len(rends) == len(ends) and all(
                np.array_equal(np.sort(fr[rends[k]:rends[k + 1]]), np.sort(order[ends[k]:ends[k + 1]]))
                for k in range(len(ends) - 1)))
    return out


def _pct(lat, q):
    return float(np.percentile(lat, q)) * 1e3 if len(lat) else None


def run_incremental(baseline=None):
    """Batched incremental sizing loop: a 200k-gate design of the small-design
    kind (designgen: 4 cell functions in drive strengths X1/X2/X4, 7x7 NLDM
    tables, 5% flops; RC trees of 2..512 nodes, log-uniform), 1000
    iterations, each resizing a random 0.5% of the gates to another drive
    strength (Timer::repower_gate) and re-timing: otg_apply_updates (new pin
    caps, new cell-arc records), otg_rc_timing_subset over the dirty nets,
    otg_propagate over the timing graph, otg_worst_slack.
      batched: all iterations' launch sets queued back to back from device
               arrays prepared before the timed region, no host round trip
               between iterations;
      plain:   the same launch set per iteration, with a synchronization and
               a read of the worst slack after each.
    Both are checked against each other iteration by iteration (worst
    slacks bit-identical).  With `baseline` (the CPU-baseline leg's dict),
    the reference Timer (oracle/_ref/ot_run_ref, CPU path, all host
    threads) runs the first INC_REF_ITERS iterations, repower_gate per gate
    and update_timing per iteration, timed; every pin after them is checked
    against ours."""
    import subprocess
    import tempfile
    import torch
    from opentimer_b200 import designgen
    from opentimer_b200.sizing import SizingDesign, resize_trace, write_ops
    out = {}
    with tempfile.TemporaryDirectory() as d:
        keep = {}
        t0 = time.perf_counter()
        info = designgen.write_design(d, seed=SEED + 3, gates=INC_GATES, keep=keep,
                                      rc_nodes=(2, 512), rc_log=True)
        t_gen = time.perf_counter() - t0
        k = int(round(INC_FRAC * INC_GATES))
        steps = resize_trace(keep, SEED + 5, INC_ITERS, k)
        t0 = time.perf_counter()
        sd = SizingDesign(d, keep)
        sd.check()
        t_load = time.perf_counter() - t0
        t0 = time.perf_counter()
        prep = sd.prepare(steps)
        t_prep = time.perf_counter() - t0
        dirty = np.diff(prep["o_net"])
        V = sd.batch.total_nodes
        # warm-up: an empty batch through the whole launch set
        for _ in range(3):
            sd.resize([])
        sd.check()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record()
        sd.run_prepared(prep)
        ev[1].record()
        torch.cuda.synchronize()
        ms_b = ev[0].elapsed_time(ev[1]) / INC_ITERS
        sd.check()
        wns_b = prep["wns"].cpu().numpy()
        del sd, prep
        torch.cuda.empty_cache()
        # plain path on a fresh copy of the design, the first iterations
        n_p = min(INC_PLAIN_ITERS, INC_ITERS)
        sp = SizingDesign(d, keep)
        prep_p = sp.prepare(steps[:n_p])
        for _ in range(3):
            sp.resize([])
        sp.check()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        wns_p = sp.run_prepared(prep_p, sync_each=True)
        ms_p = 1e3 * (time.perf_counter() - t0) / n_p
        same = bool(np.array_equal(np.array(wns_p), wns_b[:n_p]))
        out = {"workload": f"{info['gates']} gates, {info['nets']} nets, {V} RC nodes "
                           f"(trees 2..512, log-uniform), {sp.P} pins, {sp.graph.A} arcs, "
                           f"{sp.graph.num_levels} levels; {INC_ITERS} iterations x {k} gate "
                           f"resizes (0.5%)",
               "batched": {"ms_per_iteration": ms_b, "gate_resizes_per_s": k / (ms_b / 1e3),
                           "path": "iterations queued back to back: otg_apply_updates, "
                                   "otg_rc_timing_subset (dirty nets), otg_propagate, "
                                   "otg_worst_slack; device-resident design"},
               "plain": {"ms_per_iteration": ms_p, "gate_resizes_per_s": k / (ms_p / 1e3),
                         "iterations_timed": n_p,
                         "path": "the same launch set per iteration, then a synchronization "
                                 "and a read of its worst slack"},
               "speedup_vs_plain": ms_p / ms_b,
               "dirty_nets_per_iteration": float(dirty.mean()),
               "worst_slack_batched_equals_plain": same,
               "worst_slack_first_last": [wns_b[0].tolist(), wns_b[-1].tolist()],
               "design_write_s": t_gen, "design_load_s": t_load, "prepare_s": t_prep}
        exe = os.path.join(ROOT, "oracle", "_ref", "ot_run_ref")
        if baseline is not None and os.path.exists(exe):
            # ours after INC_REF_ITERS iterations: the plain copy, rebuilt
            del sp, prep_p
            torch.cuda.empty_cache()
            sr = SizingDesign(d, keep)
            for st in steps[:INC_REF_ITERS]:
                sr.resize(st)
            ours = sr.pins()
            ops = os.path.join(d, "ops.txt")
            write_ops(ops, steps[:INC_REF_ITERS])
            ref_out = os.path.join(d, "ref.txt")
            p = subprocess.run([exe, d, "cpu", ref_out, f"repower={ops}",
                                f"dump_every={INC_REF_ITERS}"], capture_output=True, text=True,
                               timeout=900)
            secs = [float(x.split()[2]) for x in p.stdout.splitlines()
                    if x.startswith("repower_step_s")]
            if p.returncode == 0 and secs:
                sys.path.insert(0, os.path.join(ROOT, "tests"))
                from helpers import pin_err, read_ref_pins
                ref = read_ref_pins(f"{ref_out}.step{INC_REF_ITERS}")
                baseline["incremental"] = {
                    "value": 1e3 * float(np.mean(secs)), "unit": "ms per iteration",
                    "cores": os.cpu_count(), "kind": "reference",
                    "sample": f"the first {INC_REF_ITERS} of the {INC_ITERS} iterations",
                    "what": "the reference Timer (oracle/_ref): repower_gate per resized gate, "
                            "then update_timing (dirty nets and the affected cone), CPU path",
                    "ours_pins_err_over_tol": pin_err(ours, ref)}
                out["reference_ms_per_iteration"] = 1e3 * float(np.mean(secs))
                out["speedup_vs_reference"] = 1e3 * float(np.mean(secs)) / ms_b
                out["pins_err_over_tol_vs_reference"] = baseline["incremental"][
                    "ours_pins_err_over_tol"]
    return out


def _served_design(args):
    """One served design, built in a worker process: its files in `d` and
    its host side (gateserve.build_design); the gates and libraries the
    request generator needs come back with it."""
    d, seed, gates = args
    sys.path.insert(0, ROOT)
    from opentimer_b200 import designgen
    from opentimer_b200.gateserve import build_design
    keep = {}
    designgen.write_design(d, seed=seed, gates=gates, keep=keep, lib_seed=SEED + 400)
    out = build_design(d, keep)
    light = {"gates": [(g, c, None) for g, c, _ in keep["gates"]], "libs": keep["libs"]}
    return out, light


def run_serving(baseline=None):
    """Served incremental timing: SRV_DESIGNS device-resident designs of the
    small-design kind (one shared cell library), pins log-uniform in
    SRV_PINS_LO..SRV_PINS_HI, held as one union on the device
    (gateserve.DesignSet).  Requests resize 1..64 random gates of one design
    (another drive strength each) and ask for its worst slack; Poisson
    streams at SRV_RATES req/s (up to SRV_MAX_REQ requests each) and a
    saturation run (SRV_SAT_REQ requests queued at once).  Batched:
    continuous batching, at most one request per design per batch, one
    launch set per batch (apply, RC over the dirty nets, propagation of the
    batch's designs only, worst slack per design).  Plain: one request at a
    time through the same launch set.  Every request's worst slack is
    checked equal on both paths.  With `baseline`, SRV_DESIGNS reference
    Timers (oracle/_ref/ot_run_ref, CPU path, one process per design, all
    at once) serve the first SRV_REF_REQ requests of every design of the
    saturation trace (repower_gate per gate, update_timing), timed."""
    import multiprocessing as mp
    import subprocess
    import tempfile
    import torch
    from concurrent.futures import ThreadPoolExecutor
    from opentimer_b200.gateserve import DesignSet, GateServer, request_trace
    from opentimer_b200.sizing import write_ops
    rng = np.random.default_rng(SEED + 7)
    pins = np.exp(rng.uniform(np.log(SRV_PINS_LO), np.log(SRV_PINS_HI), SRV_DESIGNS))
    gates = np.maximum((pins / SRV_PINS_PER_GATE).astype(np.int64), 1000)
    with tempfile.TemporaryDirectory() as root:
        dirs = [os.path.join(root, f"d{i}") for i in range(SRV_DESIGNS)]
        t0 = time.perf_counter()
        order = np.argsort(-gates)  # the largest designs first
        with mp.get_context("spawn").Pool(min(SRV_DESIGNS, os.cpu_count() or 1)) as pool:
            built = pool.map(_served_design, [(dirs[i], SEED + 100 + int(i), int(gates[i]))
                                              for i in order.tolist()], chunksize=1)
        designs, keeps = [None] * SRV_DESIGNS, [None] * SRV_DESIGNS
        for k, i in enumerate(order.tolist()):
            designs[i], keeps[i] = built[k]
        t_build = time.perf_counter() - t0
        ds = DesignSet(designs)
        out = {"workload": f"{SRV_DESIGNS} designs, {ds.P} pins, {ds.graph.A} arcs, "
                           f"{ds.batch.num_nets} nets, {ds.batch.total_nodes} RC nodes; "
                           "requests resize 1..64 gates and ask for the worst slack",
               "levels": ds.graph.num_levels, "designs_build_s": t_build, "rates": []}
        srv = GateServer(ds)
        # warm-up: a few requests through both paths
        warm = request_trace(keeps, SEED + 8, 40, None, at_zero=True)
        srv.replay(warm)
        srv.replay(warm, plain=True)
        for rate in SRV_RATES:
            n = min(SRV_MAX_REQ, max(300, int(rate * 3)))  # about 3 s of arrivals
            tr = request_trace(keeps, SEED + int(rate), n, rate)
            lat_b, span_b, _ = srv.replay(tr)
            lat_p, span_p, _ = srv.replay(tr, plain=True)
            out["rates"].append({
                "offered_req_per_s": rate, "requests": n,
                "batched": {"p50_ms": _pct(lat_b, 50), "p99_ms": _pct(lat_b, 99),
                            "req_per_s": n / span_b},
                "plain": {"p50_ms": _pct(lat_p, 50), "p99_ms": _pct(lat_p, 99),
                          "req_per_s": n / span_p}})
        # saturation, and the results of the two paths on the same states:
        # two fresh copies of the designs take the same trace
        n = SRV_SAT_REQ
        tr = request_trace(keeps, SEED + 9, n, None, at_zero=True)
        del srv, ds
        torch.cuda.empty_cache()
        ds = DesignSet(designs)  # fresh: every gate back at its initial cell
        srv = GateServer(ds)
        _, span_b, res_b = srv.replay(tr)
        del srv, ds
        torch.cuda.empty_cache()
        ds = DesignSet(designs)
        srv = GateServer(ds)
        _, span_p, res_p = srv.replay(tr, plain=True)
        out["saturation"] = {"requests": n, "batched_req_per_s": n / span_b,
                             "plain_req_per_s": n / span_p, "speedup": span_p / span_b,
                             "results_equal_alone_and_mixed": bool(
                                 np.array_equal(res_b.view(np.int32), res_p.view(np.int32)))}
        exe = os.path.join(ROOT, "oracle", "_ref", "ot_run_ref")
        if baseline is not None and os.path.exists(exe):
            def ref_one(i):
                mine = [k for k in range(n) if tr["design"][k] == i][:SRV_REF_REQ]
                if not mine:
                    return None
                ops = os.path.join(dirs[i], "ops.txt")
                write_ops(ops, [tr["resizes"][k] for k in mine])
                p = subprocess.run([exe, dirs[i], "cpu", os.path.join(dirs[i], "ref.txt"),
                                    f"repower={ops}"], capture_output=True, text=True,
                                   timeout=1200)
                if p.returncode != 0:
                    return None
                return [float(x.split()[2]) for x in p.stdout.splitlines()
                        if x.startswith("repower_step_s")]
            with ThreadPoolExecutor(SRV_DESIGNS) as ex:
                steps = [x for x in ex.map(ref_one, range(SRV_DESIGNS)) if x]
            if steps:
                allst = np.concatenate(steps)
                busiest = max(sum(x) for x in steps)
                baseline["serving"] = {
                    "value": len(allst) / busiest, "unit": "requests/s",
                    "cores": os.cpu_count(), "kind": "reference",
                    "sample": f"the first {SRV_REF_REQ} requests of every design of the "
                              "saturation trace, the designs' Timers running at once",
                    "service_p50_ms": _pct(allst, 50), "service_p99_ms": _pct(allst, 99),
                    "what": "one reference Timer per design (oracle/_ref, CPU path): "
                            "repower_gate per resized gate, then update_timing"}
                out["reference_req_per_s"] = len(allst) / busiest
                out["speedup_vs_reference"] = (n / span_b) / (len(allst) / busiest)
    return out


def run_spef(baseline=None):
    """SPEF ingestion: a seeded 20k-net SPEF (2..512 nodes per net, ~1.8M
    nodes) read into the flat RC layout by otg_spef_read (all host threads,
    and one).  With `baseline` (the CPU-baseline leg's dict), the
    reference's SPEF parser plus the flat id rule (oracle/_ref, one thread,
    as the reference reads SPEF) is timed on the same file into
    baseline["spef_ingest"]."""
    import tempfile
    from opentimer_b200 import synth_forest_host, workloads
    from opentimer_b200.spef import read_spef
    ns = workloads.net_sizes(SEED + 20, SPEF_NETS, 2, 512)
    forest = synth_forest_host(SEED + 20, ns)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "forest.spef")
        V = workloads.write_spef(path, forest)
        mb = os.path.getsize(path) / 1e6

        def best(fn, reps=3):
            t = 1e30
            for _ in range(reps):
                t0 = time.perf_counter()
                fn()
                t = min(t, time.perf_counter() - t0)
            return t
        t_all = best(lambda: read_spef(path, threads=0, names=False))
        t_one = best(lambda: read_spef(path, threads=1, names=False))
        got = read_spef(path, names=False)
        same = bool(np.array_equal(got["edges"], forest["edges"]) and
                    np.array_equal(got["roots"], forest["roots"]))
        if baseline is not None and os.path.exists(os.path.join(ROOT, "oracle", "_ref",
                                                               "libotref.so")):
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O
            L = O.ref_lib()
            n, v = ctypes.c_int(), ctypes.c_int()
            t_ref = best(lambda: L.otref_spef_load(path.encode(), ctypes.byref(n),
                                                   ctypes.byref(v)), reps=1)
            baseline["spef_ingest"] = {
                "value": V / t_ref, "unit": "nodes/s", "cores": 1, "kind": "reference",
                "sample": f"the same {mb:.0f} MB file, one pass",
                "what": "the reference's SPEF parser (PEGTL) + the flat id rule"}
    return {"workload": f"{SPEF_NETS} nets, {V} nodes, {mb:.0f} MB of SPEF text",
            "nodes_per_s": V / t_all, "threads": os.cpu_count(),
            "single_thread_nodes_per_s": V / t_one, "ids_round_trip": same}


def pin_err(got, ref):
    """Worst |got - ref| / (1e-5 s + 1e-5) over pins and quantities ([4,4]:
    at, slew, rat, slack by corner), s = |ref| for at and slew and
    max(|ref|, |ref at|) for rat and slack, differences of path-length
    quantities (inf where one side has a value the other lacks)."""
    worst = 0.0
    for name, r in ref.items():
        g = got[name]
        m = ~np.isnan(r)
        if not np.array_equal(m, ~np.isnan(g)):
            return float("inf")
        scale = np.abs(r)
        scale[2:] = np.maximum(scale[2:], np.nan_to_num(np.abs(r[0])))
        if m.any():
            worst = max(worst, float(np.max(np.abs(g[m] - r[m]) / (1e-5 * scale[m] + 1e-5))))
    return worst


def run_full_update(dump=None, baseline=None):
    """A full timing update on the GPU for a seeded gate-level design
    (designgen: 4-cell library with 7x7 NLDM tables, a random DAG with 5%
    flops, one RC tree per net): SPEF read into the flat layout, the fused
    RC pass, and levelized propagation of slew/delay/arrival/required time
    and slack over the design's timing graph.  With `baseline` (the
    CPU-baseline leg's dict), the reference Timer's own update_timing on the
    same files (oracle/_ref/ot_run_ref: its CPU path on all host threads,
    and its CUDA path) is timed into baseline["full_update"], and every
    pin's results are checked against it.  Levelization, which the Timer
    redoes after a topology change, is timed apart: levelize_ms is the
    otg_levelize launch, levelize_input_build_ms the device build of its
    input (otg_fanin_csr); gpu_ms_with_levelize counts both."""
    import subprocess
    import tempfile
    import torch
    import opentimer_b200 as otg
    from opentimer_b200 import designgen
    from opentimer_b200.prop import TimingGraph, attach_nets, rc_inputs
    from opentimer_b200.spef import read_spef
    out = {}
    with tempfile.TemporaryDirectory() as d:
        keep = {}
        info = designgen.write_design(d, seed=SEED + 30, gates=FU_GATES, keep=keep)
        arrays, names, nets = designgen.timing_graph(keep)
        caps = designgen.pin_caps(keep)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        t0 = time.perf_counter()
        f = read_spef(os.path.join(d, "design.spef"), r_scale=np.float32(1e-3))
        t_spef = time.perf_counter() - t0
        cap, node_of = rc_inputs(f, caps)
        graph = TimingGraph(attach_nets(arrays, names, nets, f, node_of))
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
        batch = otg.RcBatch(t(f["nodes_start"]), t(f["edges"].copy()), t(f["roots"]),
                            t(f["res"]), t(cap))
        for _ in range(3):  # warm-up
            batch.run()
            graph.propagate(batch)
        graph.check()
        rc_t, prop_t = [], []
        for _ in range(FU_REPS):
            torch.cuda.synchronize()
            ev[0].record()
            batch.run()
            ev[1].record()
            graph.propagate(batch)
            ev[2].record()
            torch.cuda.synchronize()
            rc_t.append(ev[0].elapsed_time(ev[1]))
            prop_t.append(ev[1].elapsed_time(ev[2]))
        batch.check()
        lv_t, csr_t = [], []
        for _ in range(FU_REPS):  # levelization, as update_timing redoes it after a topology
            # change: its input built on the device (otg_fanin_csr, which
            # synchronizes for the sizes), then otg_levelize
            torch.cuda.synchronize()
            ev[0].record()
            lb = otg.LevelizeBatch(*graph.levelize_input())
            ev[1].record()
            lb.run()
            ev[2].record()
            torch.cuda.synchronize()
            lv_t.append(ev[1].elapsed_time(ev[2]))  # the levelization launch
            csr_t.append(ev[0].elapsed_time(ev[1]))  # its input, built on the device
        lb.check()
        res = graph.result()
        res["rat"] = np.where(np.isnan(res["at"]), np.nan, res["rat"])
        rc_ms, prop_ms = float(np.median(rc_t)), float(np.median(prop_t))
        lv_ms, csr_ms = float(np.median(lv_t)), float(np.median(csr_t))
        out = {"workload": f"{info['gates']} gates, {info['nets']} nets, {graph.P} pins, "
                           f"{graph.A} arcs, {graph.num_levels} levels",
               "gpu_ms": rc_ms + prop_ms, "rc_pass_ms": rc_ms, "propagation_ms": prop_ms,
               "levelize_ms": lv_ms, "levelize_input_build_ms": csr_ms,
               "gpu_ms_with_levelize": rc_ms + prop_ms + lv_ms + csr_ms,
               "timed": f"median of {FU_REPS}", "spef_read_ms": 1e3 * t_spef,
               "levels": graph.num_levels, "launches_per_propagation": 2}
        exe = os.path.join(ROOT, "oracle", "_ref", "ot_run_ref")
        if baseline is not None and os.path.exists(exe):
            ours = {n: np.stack([res[k][i] for k in ("at", "slew", "rat", "slack")])
                    for i, n in enumerate(names)}
            ref = {}
            for mode in ("cpu", "cuda"):
                ref_out = os.path.join(d, f"ref_{mode}.txt")
                p = subprocess.run([exe, d, mode, ref_out], capture_output=True, text=True,
                                   timeout=600)
                secs = [float(x.split()[1]) for x in p.stdout.splitlines()
                        if x.startswith("update_timing_s")]
                if p.returncode != 0 or not secs:
                    continue
                pins = {}
                with open(ref_out) as fh:
                    for line in fh:
                        if line.startswith("P "):
                            tk = line.split()
                            pins[tk[1]] = np.array([float(x) for x in tk[2:]]).reshape(4, 4)
                ref[mode] = (1e3 * secs[0], pins)
            if dump is not None:  # the raw results, for a caller's own analysis
                dump.update(names=names, ours=ours, ref={k: v[1] for k, v in ref.items()},
                            order=graph.order.cpu().numpy(),
                            level_ends=graph.level_ends.cpu().numpy())
            b = {}
            if "cpu" in ref:
                b.update(value=ref["cpu"][0], unit="ms per update_timing", cores=os.cpu_count(),
                         kind="reference", sample="the same design files, one full update",
                         what="the reference Timer's update_timing (oracle/_ref), CPU path")
                b["ours_pins_err_over_tol"] = pin_err(ours, ref["cpu"][1])
            if "cuda" in ref:
                b["reference_cuda_path_ms"] = ref["cuda"][0]
                b["ours_pins_err_over_tol_vs_cuda_path"] = pin_err(ours, ref["cuda"][1])
                if "cpu" in ref:
                    # the reference's own two paths against each other, same tolerance
                    b["reference_cuda_vs_cpu_pins_err_over_tol"] = pin_err(ref["cuda"][1],
                                                                           ref["cpu"][1])
            baseline["full_update"] = b
        out["incremental_spef"] = _incremental_spef(d, keep, f, caps, batch, graph, names,
                                                    baseline)
    return out


def _incremental_spef(d, keep, f0, caps, batch, graph, names, baseline=None):
    """A change SPEF (TAU15 change_*.spef style) re-drawing FU_CHANGE of the
    design's nets, applied to the device-resident design: the host reads
    the file and maps its nets and pins, then RcBatch.replace_nets moves
    the unchanged nets with their results into the new layout, re-times
    the changed nets, and the propagation runs again.  With `baseline`, the
    reference Timer's read_spef + update_timing on the same change
    (oracle/_ref, CPU path) is timed into baseline["incremental_spef"] and
    every pin is checked against it."""
    import subprocess
    import torch
    from opentimer_b200 import designgen
    from opentimer_b200.prop import change_arcs, change_nets
    from opentimer_b200.spef import read_spef
    path = os.path.join(d, "change.spef")
    changed = designgen.change_spef(keep, path, frac=FU_CHANGE, seed=SEED + 31)
    # design state kept between changes, as the Timer keeps its net map
    index = {n: i for i, n in enumerate(f0["net_names"])}
    host_t = []
    for _ in range(FU_REPS):  # the host part is repeatable: median of FU_REPS
        t0 = time.perf_counter()
        fc = read_spef(path, r_scale=np.float32(1e-3))
        nets, forest, node_of = change_nets(fc, index, caps)
        # net arcs into the changed nets get their sinks' new local ids
        sel, nodes = change_arcs(graph.net_arcs, graph.arc_to, names, nets, node_of)
        host_t.append(1e3 * (time.perf_counter() - t0))
    host_ms = float(np.median(host_t))
    forest_d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in forest]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    mv_t, pr_t = [], []
    for r in range(3 + FU_REPS):
        torch.cuda.synchronize()
        ev[0].record()
        b1 = batch.replace_nets(nets, *forest_d)
        graph.set_arc_nodes(sel, nodes)
        ev[1].record()
        graph.propagate(b1)
        ev[2].record()
        torch.cuda.synchronize()
        if r >= 3:
            mv_t.append(ev[0].elapsed_time(ev[1]))
            pr_t.append(ev[1].elapsed_time(ev[2]))
    b1.check()
    res = graph.result()
    res["rat"] = np.where(np.isnan(res["at"]), np.nan, res["rat"])
    mv_ms, pr_ms = float(np.median(mv_t)), float(np.median(pr_t))
    out = {"workload": f"change SPEF re-drawing {len(changed)} of {len(index)} nets "
                       f"({int(np.diff(forest[0]).sum())} nodes)",
           "host_read_and_map_ms": host_ms, "replace_nets_ms": mv_ms, "propagation_ms": pr_ms,
           "total_ms": host_ms + mv_ms + pr_ms, "timed": f"median of {FU_REPS}",
           "replace_nets": "relayout (otg_rc_move_nets) + subset RC pass on the changed nets"}
    exe = os.path.join(ROOT, "oracle", "_ref", "ot_run_ref")
    if baseline is not None and os.path.exists(exe):
        ref_out = os.path.join(d, "ref_change.txt")
        p = subprocess.run([exe, d, "cpu", ref_out, f"change={path}"], capture_output=True,
                           text=True, timeout=600)
        secs = [float(x.split()[1]) for x in p.stdout.splitlines()
                if x.startswith("incremental_update_timing_s")]
        if p.returncode == 0 and secs:
            pins = {}
            with open(ref_out) as fh:
                for line in fh:
                    if line.startswith("P "):
                        tk = line.split()
                        pins[tk[1]] = np.array([float(x) for x in tk[2:]]).reshape(4, 4)
            ours = {n: np.stack([res[k][i] for k in ("at", "slew", "rat", "slack")])
                    for i, n in enumerate(names)}
            baseline["incremental_spef"] = {
                "value": 1e3 * secs[0], "unit": "ms per change", "cores": os.cpu_count(),
                "kind": "reference", "sample": "the same change SPEF, one application",
                "what": "the reference Timer (oracle/_ref): read_spef(change) + update_timing, "
                        "CPU path, dirty nets only",
                "ours_pins_err_over_tol": pin_err(ours, pins)}
    return out


def run_huge():
    """Nets above the shared-memory classes (the seeded generator's trees
    and chains at 20k and 5k-20k nodes): the cluster path (one thread-block
    cluster of 8 CTAs per net, chosen on the device when there are at most
    two nets per cluster) against one CTA per net over a workspace slice
    (OTG_RC_HUGE_CLUSTER=1), CUDA events, median of 5 passes after 2; the
    two paths' outputs are compared bit for bit."""
    import torch
    import opentimer_b200 as otg
    from opentimer_b200 import workloads
    out = {}
    cases = [("8 nets x 20000 nodes", np.arange(9, dtype=np.int32) * 20000),
             ("1 net x 20000 nodes", np.array([0, 20000], np.int32)),
             ("200 nets, 5000..20000 nodes", workloads.net_sizes(SEED + 11, 200, 5000, 20000))]
    for name, ns_np in cases:
        ns = torch.from_numpy(ns_np).cuda()
        g = otg.synth_forest(SEED + 11, ns)
        V = int(ns_np[-1])
        res, outs = {}, {}
        for path, env in (("one_cta_per_net", "1"), ("default", None)):
            if env is None:
                os.environ.pop("OTG_RC_HUGE_CLUSTER", None)
            else:
                os.environ["OTG_RC_HUGE_CLUSTER"] = env
            try:
                b = otg.RcBatch(ns, g["edges"].clone(), g["roots"], g["res"], g["cap"],
                                max_net_nodes=int(np.diff(ns_np).max()))
                for _ in range(2):
                    b.run()
                b.check()
                times = []
                for _ in range(5):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record()
                    b.run()
                    e1.record()
                    torch.cuda.synchronize()
                    times.append(e0.elapsed_time(e1))
                b.check()
                ms = float(np.median(times))
                res[path] = {"ms": ms, "nodes_per_s": V / ms * 1e3}
                outs[path] = [getattr(b, q).cpu() for q in ("node2bfs", "pid", "load", "delay",
                                                             "ldelay", "impulse")]
                del b
            finally:
                os.environ.pop("OTG_RC_HUGE_CLUSTER", None)
        res["speedup"] = res["one_cta_per_net"]["ms"] / res["default"]["ms"]
        res["outputs_identical"] = all(torch.equal(x, y) for x, y in
                                       zip(outs["one_cta_per_net"], outs["default"]))
        out[name] = res
    out["what"] = ("default: clusters of 8 CTAs per net when the device-side count of huge nets "
                   "is at most 2 per cluster, else one CTA per net")
    return out


def reference_gpu_rc(ns_np, seed, budget_s=8.0):
    """The reference's own sm_100a RC kernels (rct_bfs_and_compute_cuda,
    ot/cuda/rct.cu:361-397, oracle/_ref) on the first nets of the headline
    workload: the whole call as the Timer makes it (host arrays, its own
    allocations and copies) and its kernels alone (CUDA events around each
    of its launches), next to our fused pass on the very same nets.  The
    sample is sized from a timed 300-net prefix to about `budget_s` of the
    reference's time; its chains stay in (its BFS costs depth x edges per
    net, which is the point of the comparison).  Its BFS slots and pid are
    compared with ours."""
    import torch
    import opentimer_b200 as otg
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available():
        return {"error": "oracle/_ref not built"}
    ns64 = ns_np.astype(np.int64)

    def sample(k):
        f, slew, _ = O.synth_forest(seed, ns64[:k + 1], threads=os.cpu_count())
        return f
    O.ref_rct_gpu(sample(50))  # context, module load
    t = {}
    f = sample(300)
    O.ref_rct_gpu(f, timing=t)
    k = int(min(len(ns64) - 1, max(300, 300 * budget_s / max(t["call_s"], 1e-3))))
    k = min(k, 200_000)
    f = sample(k)
    t = {}
    e_ref, n2b_ref, pid_ref, _ = O.ref_rct_gpu(f, timing=t)
    V = f.total_nodes
    # ours on the same nets, device-resident inputs
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    b = otg.RcBatch(d(f.nodes_start), d(f.edges.copy()), d(f.roots), d(f.res), d(f.cap),
                    max_net_nodes=int(np.diff(ns64[:k + 1]).max()))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ts = []
    for r in range(6):
        torch.cuda.synchronize()
        ev[0].record()
        b.run()
        ev[1].record()
        torch.cuda.synchronize()
        if r:
            ts.append(ev[0].elapsed_time(ev[1]))
    b.check()
    ours_ms = float(np.median(ts))
    nonroot = np.ones(V, bool)
    nonroot[f.nodes_start[:-1]] = False  # the reference leaves a net's root pid unwritten
    same = bool(np.array_equal(b.node2bfs.cpu().numpy(), n2b_ref) and
                np.array_equal(b.pid.cpu().numpy()[nonroot], pid_ref[nonroot]))
    del b
    torch.cuda.empty_cache()
    return {"sample": f"first {k} of the {len(ns64) - 1} headline nets ({V} nodes)",
            "reference_call_nodes_per_s": V / t["call_s"],
            "reference_call_ms": 1e3 * t["call_s"],
            "reference_kernel_ms": t["kernel_ms"], "reference_kernel_launches": t["launches"],
            "reference_kernel_nodes_per_s": V / (t["kernel_ms"] / 1e3),
            "ours_pass_ms": ours_ms, "ours_nodes_per_s": V / (ours_ms / 1e3),
            "kernel_speedup": t["kernel_ms"] / ours_ms,
            "bfs_slots_match_reference_gpu": same,
            "what": "reference: rct_bfs_and_compute_cuda built -arch sm_100a (oracle/_ref); "
                    "kernel time = CUDA events around its compute_net_bfs, prepare_res_cap "
                    "and compute_net_timing launches; ours: otg_rc_timing on device inputs, "
                    "median of 5"}


def cpu_baseline(g, ns_np):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    threads = os.cpu_count() or 1
    rate = calibrate_cpu(lambda k: cpu_sample(ns_np, g, k), ns_np, threads)
    k = sample_nets_for_budget(ns_np, 15.0, rate)
    f = cpu_sample(ns_np, g, k)
    dt, kind, cores = time_reference_cpu(f, threads)
    return {"value": f.total_nodes / dt, "unit": "nodes/s", "cores": cores, "kind": kind,
            "sample": f"first {k} of {NUM_NETS} nets ({f.total_nodes} nodes), one pass"}


T_START = time.perf_counter()


def main():
    global INC_GATES, INC_ITERS, SRV_DESIGNS, SRV_PINS_HI
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-levelize", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-incremental", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--tuning", default=None,
                    help="RC-pass tuning to apply instead of autotuning (JSON or a JSON file)")
    ap.add_argument("--no-spef", action="store_true")
    ap.add_argument("--no-full-update", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--no-huge", action="store_true")
    ap.add_argument("--inc-gates", type=int, default=INC_GATES,
                    help="gates of the incremental sizing loop's design (smaller: quick runs)")
    ap.add_argument("--inc-iters", type=int, default=INC_ITERS)
    ap.add_argument("--srv-designs", type=int, default=SRV_DESIGNS,
                    help="served designs (smaller: quick runs)")
    ap.add_argument("--srv-pins-hi", type=int, default=SRV_PINS_HI)
    # smaller cases (profiling); the defaults are the benchmark workload
    ap.add_argument("--nets", type=int, default=NUM_NETS)
    ap.add_argument("--min-nodes", type=int, default=2)
    ap.add_argument("--max-nodes", type=int, default=4096)
    args = ap.parse_args()
    INC_GATES, INC_ITERS = args.inc_gates, args.inc_iters
    SRV_DESIGNS, SRV_PINS_HI = args.srv_designs, args.srv_pins_hi
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            line = run_ours(args, world, rank, local)
            if rank == 0:
                print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
