"""Benchmark of the Louvain hot path: edges/s per Louvain pass.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload rmat25|lfr|sbm10k|rmat<scale>|batched|serving]
                    [--impl ours|reference] [--graphs G]

Workload (default): the R-MAT graph of scale 25 (33,554,432 vertices, edge
factor 16, (a,b,c,d) = (0.57, 0.19, 0.19, 0.05), self loops dropped,
duplicates merged by summing weights, integer weights 1..16, seed 2;
1,047,217,118 symmetric entries) -- synthetic, seeded; generated on the
device for the GPU arm and by the same generator on the host for the
reference arm (the two are equal entry for entry).

One step (value) = the move passes of the level-0 one-level phase: both
passes (the singleton pass and the hashing pass), the ΔQ test, commit and
isolated-vertex merge on the device-resident CSR.  value = CSR entries x
passes / step time.  e2e = one whole dendrogram run through the C ABI from
pinned host buffers: H2D of the edge list, CSR build, every level, final FP64
modularity and D2H of the partition; e2e value = sum over levels of CSR
entries x passes / run time.

--impl reference times the oracle (the CPU restatement of the reference's
method) on the same graph and the same two passes, on all host cores: each
step decides a bounded sample of the vertices (every 8th vertex, a different
eighth per step) from the singleton state and from the state after a full
first pass; value = sampled CSR entries x 2 / decision time.

With --gpus N each rank runs an independent replica (the path does not shard
within one graph); value is the sum over ranks of entries processed divided by
the slowest rank's time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edges/s per Louvain pass"
DEVICE_GEN_SCALE = 20     # R-MAT graphs this large are generated on the device
UNIT = "edges/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="rmat25")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default degree thresholds instead of tuning them on the workload graph")
    ap.add_argument("--thresholds", default="",
                    help="TILE,BLOCK: run with these degree thresholds instead of tuning (profiling runs)")
    ap.add_argument("--graphs", type=int, default=8192, help="batched workload: number of graphs")
    ap.add_argument("--batch-entries", type=float, default=1.25e8,
                    help="batched/serving workloads: entries per packed sub-batch")
    ap.add_argument("--batch-workers", type=int, default=4,
                    help="batched workload: contexts running sub-batches at the same time")
    ap.add_argument("--requests", type=int, default=5000, help="serving workload: requests")
    ap.add_argument("--rate", type=float, default=2000.0, help="serving workload: Poisson arrivals per second")
    ap.add_argument("--pool", type=int, default=2048, help="serving workload: distinct small graphs")
    ap.add_argument("--giants", type=int, default=4, help="serving workload: distinct R-MAT scale-22 graphs")
    ap.add_argument("--slots", type=int, default=4, help="serving workload: server slots")
    return ap.parse_args()


def make_graph(workload, host=False):
    """(n, src, dst, w, config description, level gain threshold) of a plain
    workload; R-MAT graphs of scale >= DEVICE_GEN_SCALE are generated on the
    device unless `host` (the reference arm, which runs no device code)."""
    from louvaingpu_b200 import graphgen
    if workload == "lfr":
        n, s, d, w = graphgen.lfr()
        desc = dict(workload="LFR-style power-law graph", n_vertices=n, degree_exp=2.5, degree_range=[5, 5000],
                    community_exp=1.5, community_range=[50, 50000], mu=0.3, weights="unit", seed=1)
        return n, s, d, w, desc, 1e-7
    if workload == "sbm10k":
        n, s, d, w = graphgen.sbm_10k(seed=0)
        desc = dict(workload="planted-partition SBM", n_vertices=n, blocks=100, p_in=0.1, p_out=0.0006,
                    weights="unit", seed=0, level_min_gain=1e-6)
        return n, s, d, w, desc, 1e-6
    if workload.startswith("rmat"):
        scale = int(workload[4:])
        if scale >= DEVICE_GEN_SCALE and not host:
            # generated on the device (equal to the host generator), copied back once
            dg = graphgen.rmat_device(scale)
            n = dg.n_vertices
            s, d, w = dg.to_host()
            dg.close()
        else:
            n, s, d, w = graphgen.rmat(scale)
        desc = dict(workload=f"R-MAT scale {scale}", n_vertices=n, edge_factor=16, abcd=[0.57, 0.19, 0.19, 0.05],
                    self_loops="dropped", duplicates="merged, weights summed", weights="integer 1..16", seed=2,
                    label_noise="none")
        return n, s, d, w, desc, 1e-7
    raise SystemExit(f"unknown workload {workload}")


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(workload):
    """DRAM bytes per move pass from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "move_pass_traffic.json")
    try:
        with open(p) as f:
            j = json.load(f)
        return j.get(workload)
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"lvg_bench_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            t0 = time.time()
            while time.time() - t0 < 5.0:   # wait for the first sample before timing starts
                time.sleep(0.05)
                if os.path.getsize(self.path) > 0:
                    break
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
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def phase_roofline(levels, peak):
    """Algorithmic bytes and achieved GB/s of the level phases of one run, on
    the least traffic each phase needs: the CSR build reads the level list
    (12 B per entry) and writes the CSR (8 B per entry) and the per-vertex
    offsets and degrees (16 B); the coarsening reads the level list (12 B per
    entry) and writes the coarse list (12 B per coarse entry) and its CSR
    (8 B per coarse entry); renumbering reads and writes 12 B per vertex."""
    tot = {"build": 0.0, "induce": 0.0, "renumber": 0.0}
    ms = {"build": 0.0, "induce": 0.0, "renumber": 0.0}
    for l, x in enumerate(levels):
        tot["build"] += 20.0 * x.n_entries + 16.0 * x.n_vertices
        ms["build"] += x.ms_build
        tot["renumber"] += 12.0 * x.n_vertices
        ms["renumber"] += x.ms_renumber
        if l + 1 < len(levels):
            tot["induce"] += 12.0 * x.n_entries + 20.0 * levels[l + 1].n_entries
            ms["induce"] += x.ms_induce
    out = {}
    for k in tot:
        gbs = tot[k] / (ms[k] * 1e-3) / 1e9 if ms[k] > 0 else 0.0
        out[k] = {"algorithmic_bytes": tot[k], "ms": round(ms[k], 3), "achieved_gbs": round(gbs, 1),
                  "frac": round(gbs / peak, 4)}
    return out


SAMPLE_STRIDE = 8        # CPU legs: every 8th vertex per step
STEP = "move passes of the level-0 one-level phase (singleton pass + hashing pass)"


class CpuPassSample:
    """The two level-0 move passes run by the oracle (the CPU restatement of
    the reference's method, OneLevelKernel.cu:248-422) on the workload graph,
    over a bounded sample per step: the vertices i with i % 8 == step % 8
    (every eighth vertex, a different eighth each step), decided from the
    singleton state (pass 1) and from the state after a full first pass
    (pass 2), as the one-level phase runs them.  The full first pass that
    sets up pass 2 runs once, untimed."""

    def __init__(self, n, s, d, w, threads):
        from oracle import oracle as O
        self.threads = threads
        self.c = O.Csr(n, s, d, w, arrays=False)
        V = self.c.V
        self.deg = np.diff(self.c.off)
        self.state0 = (np.arange(V, dtype=np.int32), self.c.k, np.ones(V, np.int32))
        nxt = self.c.decide(*self.state0, n_threads=threads)[0]
        tot = np.bincount(nxt, weights=self.c.k, minlength=V)   # integral weights: exact in any order
        self.state1 = (nxt, tot, np.bincount(nxt, minlength=V).astype(np.int32))

    def step(self, k):
        """(entries decided, seconds) of one step: both passes over sample k."""
        verts = np.arange(k % SAMPLE_STRIDE, self.c.V, SAMPLE_STRIDE, dtype=np.int32)
        t1, _ = self.c.decide_subset(*self.state0, verts, n_threads=self.threads)
        t2, _ = self.c.decide_subset(*self.state1, verts, n_threads=self.threads)
        return 2 * int(self.deg[verts].sum()), t1 + t2

    def sample_text(self, steps):
        return (f"{steps} steps, each both level-0 move passes of the oracle over every {SAMPLE_STRIDE}th vertex "
                f"of the workload graph (a different eighth per step), decision time only")


def plain_config(desc, E, nnz, V, gpus):
    """config of the plain workloads, the same in both arms."""
    mb = (12.0 * nnz + 24.0 * V) / 1e6
    l2 = ("inputs larger than L2 (move pass touches %.0f MB)" % mb if mb > 126.0 else
          "inputs fit in L2 (move pass touches %.1f MB; no flush between steps)" % mb)
    return dict(desc, n_entries=E, csr_entries=nnz, parallelism="replicas" if gpus > 1 else "single", step=STEP,
                l2=l2)


def max_over_ranks(values, pg):
    """Element-wise max over the ranks (device times: the slowest rank sets
    the job's time).  NCCL reduces on the GPU, gloo on the host."""
    if not pg:
        return list(values)
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def whole_job_rate(units_per_rank, world, t_max_ms):
    """Units every rank processed (equal per rank: replicas / weak scaling)
    divided by the slowest rank's time."""
    return units_per_rank * world / (t_max_ms / 1e3)


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def run_reference(args, world, rank, pg):
    """Reference arm: the CPU restatement of the reference's method (the
    reference has no CPU Louvain and its GPU code cannot be built here) on all
    host cores, on the same graph and the same two level-0 passes as the GPU
    arm, over a bounded vertex sample per step (CpuPassSample)."""
    if rank != 0:
        return
    n, s, d, w, desc, level_min = make_graph(args.workload, host=True)
    E = len(s)
    threads = os.cpu_count() or 1
    cs = CpuPassSample(n, s, d, w, threads)
    del s, d, w
    for k in range(args.warmup):
        cs.step(k)
    entries, t = 0, 0.0
    for k in range(args.steps):
        e, secs = cs.step(args.warmup + k)
        entries += e
        t += secs
    v = entries / t
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
        "config": plain_config(desc, E, cs.c.nnz, cs.c.V, args.gpus),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": cs.sample_text(args.steps) + " (CPU restatement of the reference method; the "
                                   "reference's own GPU code cannot be built here)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local, pg):
    import torch
    from louvaingpu_b200 import Louvain, kernel_launches
    torch.cuda.set_device(local)
    n, s, d, w, desc, level_min = make_graph(args.workload)
    E = len(s)
    stream = torch.cuda.current_stream()
    # ---------------------------------------------------------------- value
    ds = torch.from_numpy(s).cuda()
    dd = torch.from_numpy(d).cuda()
    dw = torch.from_numpy(w).cuda()
    lv = Louvain(device=local, level_min_gain=level_min)
    lv.set_stream(stream.cuda_stream)
    lv.load_edges_device(ds.data_ptr(), dd.data_ptr(), dw.data_ptr(), E, n)
    V, nnz, m = lv.csr_shape()
    # degree thresholds of the move kernels: tuned once on this graph, outside
    # the timed region (a shape class is tuned once per process)
    tune = {"tile_max_degree": 512, "block_max_degree": 4096, "autotuned": False}
    if args.thresholds:
        t_, b_ = (int(x) for x in args.thresholds.split(","))
        lv.close()
        lv = Louvain(device=local, level_min_gain=level_min, tile_max_degree=t_, block_max_degree=b_)
        lv.set_stream(stream.cuda_stream)
        lv.load_edges_device(ds.data_ptr(), dd.data_ptr(), dw.data_ptr(), E, n)
        tune = {"tile_max_degree": t_, "block_max_degree": b_, "autotuned": False, "given": True}
    elif not args.no_autotune:
        from louvaingpu_b200 import LvgError
        t_tune = time.perf_counter()
        try:
            best, pts = lv.autotune(reps=3)
            tune = {"tile_max_degree": best[0], "block_max_degree": best[1], "autotuned": True,
                    "tune_s": round(time.perf_counter() - t_tune, 2),
                    "points": [[p[0], p[1], round(p[2], 4)] for p in pts]}
        except LvgError as e:   # keep the default pair; the context is rebuilt at level 0 either way
            tune["autotune_error"] = str(e)
            lv.load_edges_device(ds.data_ptr(), dd.data_ptr(), dw.data_ptr(), E, n)
            tune["tile_max_degree"], tune["block_max_degree"] = lv.thresholds()
    q0 = lv.modularity()
    clocks = Clocks(local)
    clocks.start()
    for _ in range(args.warmup):
        lv.one_level(q0)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    l0 = kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    passes_total, move_ms, move_passes = 0, 0.0, 0
    per_pass = []
    for _ in range(args.steps):
        q, p = lv.one_level(q0)
        passes_total += p
        ms, mp = lv.move_stats()
        move_ms += ms
        move_passes += mp
        per_pass.append(lv.move_pass_times().tolist())
    e1.record(stream)
    torch.cuda.synchronize()
    launches = kernel_launches() - l0
    t_ms = e0.elapsed_time(e1)
    if pg:
        t_ms = max_over_ranks([t_ms], pg)[0]
    entries = nnz * passes_total
    value = whole_job_rate(entries, world, t_ms)
    # roofline of the move kernels: B_pass = 12 nnz + 24 V bytes per pass
    peak, peak_kind = measured_peak()
    b_pass = 12.0 * nnz + 24.0 * V
    t_move = move_ms / max(move_passes, 1) / 1e3
    achieved = b_pass / t_move / 1e9 if t_move > 0 else 0.0
    by_pass = [float(np.median([x[k] for x in per_pass if len(x) > k])) for k in range(max(len(x) for x in per_pass))]
    names = ["singleton (table-free) kernels", "hashing kernels"]
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_kind, "traffic": profiled_traffic(args.workload),
            "kernel": "move kernels of one pass (all degree classes), mean over the step's passes",
            "algorithmic_bytes": b_pass, "move_ms_per_pass": t_move * 1e3,
            "passes": [{"pass": k + 1, "kernels": names[min(k, 1)], "ms": round(ms, 4),
                        "achieved": round(b_pass / (ms * 1e-3) / 1e9, 1) if ms > 0 else 0.0,
                        "frac": round(b_pass / (ms * 1e-3) / 1e9 / peak, 4) if ms > 0 else 0.0}
                       for k, ms in enumerate(by_pass)]}
    del lv, ds, dd, dw
    torch.cuda.empty_cache()
    # ---------------------------------------------------------------- e2e
    hs = torch.from_numpy(s).pin_memory()
    hd = torch.from_numpy(d).pin_memory()
    hw = torch.from_numpy(w).pin_memory()
    lv2 = Louvain(device=local, level_min_gain=level_min, tile_max_degree=tune["tile_max_degree"],
                  block_max_degree=tune["block_max_degree"])
    lv2.set_stream(stream.cuda_stream)
    part = torch.empty(n, dtype=torch.int32).pin_memory()
    for _ in range(max(1, args.warmup)):
        lv2.load_edges_ptr(hs.data_ptr(), hd.data_ptr(), hw.data_ptr(), E, n)
        lv2.run()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    pe = 0
    qf = None
    for _ in range(args.steps):
        lv2.load_edges_ptr(hs.data_ptr(), hd.data_ptr(), hw.data_ptr(), E, n)
        res = lv2.run()
        lv2.partition(out=part)
        pe += res.pass_entries
        qf = res.q_final
    f1.record(stream)
    torch.cuda.synchronize()
    t2 = f0.elapsed_time(f1)
    if pg:
        t2 = max_over_ranks([t2], pg)[0]
    clk = clocks.stop()
    e2e_value = pe * world / (t2 / 1e3)
    # one more run, timed by part on the host (not part of the timed steps)
    torch.cuda.synchronize()
    h0 = time.perf_counter()
    lv2.load_edges_ptr(hs.data_ptr(), hd.data_ptr(), hw.data_ptr(), E, n)
    h1 = time.perf_counter()
    lv2.run()
    h2 = time.perf_counter()
    lv2.partition(out=part)
    h3 = time.perf_counter()
    levels = [lv2.level_info(l) for l in range(lv2.n_levels)]
    phases = {k: round(sum(getattr(x, "ms_" + k) for x in levels), 3) for k in ("build", "passes", "renumber", "induce")}
    phases.update(host_load_ms=round((h1 - h0) * 1e3, 3), host_run_ms=round((h2 - h1) * 1e3, 3),
                  host_partition_ms=round((h3 - h2) * 1e3, 3))
    phase_roof = phase_roofline(levels, measured_peak()[0])
    del lv2
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        del hs, hd, hw
        cs = CpuPassSample(n, s, d, w, threads)
        e, secs = cs.step(0)
        cpu = {"value": e / secs, "unit": UNIT, "cores": threads, "kind": "port", "sample": cs.sample_text(1)}
        del cs
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
        "config": plain_config(desc, E, nnz, V, args.gpus),
        "passes_per_step": passes_total // args.steps,
        "tuning": tune,
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 12 * E, "d2h_bytes_per_step": 4 * n,
                "ms_per_run": t2 / args.steps, "q_final": qf, "levels": len(levels),
                "phases_ms": phases, "phase_roofline": phase_roof},
        "clocks": clk,
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- batched form
def batched_plan(count, seed, max_entries):
    """The batched workload's graphs (SBM parameters) and their split into
    packed sub-batches of at most about max_entries expected entries."""
    from louvaingpu_b200 import graphgen
    params = graphgen.batched_sbm_params(count, seed=seed)
    groups, cur, acc = [], [], 0.0
    for p in params:
        n, B = p["n"], p["blocks"]
        k = np.arange(B + 1, dtype=np.int64)
        sizes = np.diff(n * k // B).astype(np.float64)
        pin = float((sizes * (sizes - 1) / 2).sum())
        e = 2.0 * (pin * min(p["p_in"], 1.0) + (n * (n - 1) / 2 - pin) * min(p["p_out"], 1.0))
        if cur and acc + e > max_entries:
            groups.append(cur)
            cur, acc = [], 0.0
        cur.append(p)
        acc += e
    if cur:
        groups.append(cur)
    return params, groups


def run_batched(args, world, rank, local, pg):
    """graphs/s of the batched form (lvg_batch_run_device over packed
    sub-batches) against the plain per-graph loop on the same GPU."""
    import torch
    from louvaingpu_b200 import Louvain, graphgen, kernel_launches
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    params, groups = batched_plan(args.graphs, 3 + rank, args.batch_entries)
    dgs = [graphgen.sbm_batch_device(g, device=local) for g in groups]
    torch.cuda.synchronize()
    G = sum(d.n_graphs for d in dgs)
    E = sum(d.n_entries for d in dgs)
    V = sum(d.n_vertices for d in dgs)
    # workers: contexts (own streams) that take the sub-batches in turn, so
    # one batch's host checks and small kernels overlap another's work
    nw = max(1, min(args.batch_workers, len(dgs)))
    # degree thresholds tuned once on the batch's largest graph (outside the
    # timed region); every worker context builds its levels with that pair
    tune = {"tile_max_degree": 512, "block_max_degree": 4096, "autotuned": False}
    if not args.no_autotune:
        big = max(((d, g) for d in dgs for g in range(d.n_graphs)), key=lambda x: x[0].graph_ptrs(x[1])[3])
        with Louvain(device=local) as tl:
            tl.load_edges_device(*big[0].graph_ptrs(big[1]))
            best, _ = tl.autotune(reps=2)
        tune = {"tile_max_degree": best[0], "block_max_degree": best[1], "autotuned": True,
                "tuned_on": "largest graph of the batch"}
    ctxs = [Louvain(device=local, tile_max_degree=tune["tile_max_degree"], block_max_degree=tune["block_max_degree"])
            for _ in range(nw)]
    if nw == 1:
        ctxs[0].set_stream(stream.cuda_stream)
    lv = ctxs[0]

    def batched_step():
        if nw == 1:
            return [lv.run_batch_device(d.src, d.dst, d.w, d.entry_off, d.vertex_off) for d in dgs]
        import threading
        out = [None] * len(dgs)
        errs = []

        def work(k):
            try:
                for b in range(k, len(dgs), nw):
                    d = dgs[b]
                    out[b] = ctxs[k].run_batch_device(d.src, d.dst, d.w, d.entry_off, d.vertex_off)
            except Exception as e:   # reported after the join
                errs.append(e)
        ts = [threading.Thread(target=work, args=(k,)) for k in range(nw)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        if errs:
            raise errs[0]
        return out

    clocks = Clocks(local)
    clocks.start()
    for _ in range(args.warmup):
        batched_step()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    l0 = kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        res = batched_step()
    e1.record(stream)
    torch.cuda.synchronize()
    launches = kernel_launches() - l0
    t_ms = e0.elapsed_time(e1)
    # plain loop: one context, one graph at a time, same device-resident lists
    pl = Louvain(device=local, tile_max_degree=tune["tile_max_degree"], block_max_degree=tune["block_max_degree"])
    pl.set_stream(stream.cuda_stream)
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    mism, dq_max = 0, 0.0
    plain_q = []
    for d, r in zip(dgs, res):
        for g in range(d.n_graphs):
            sp, dp, wp, e, n = d.graph_ptrs(g)
            pl.load_edges_device(sp, dp, wp, e, n)
            rr = pl.run()
            part = pl.partition()
            plain_q.append(rr.q_final)
            if not np.array_equal(part, r.part(g)):
                mism += 1
            dq_max = max(dq_max, abs(rr.q_final - r.q_final[g]))
    p1.record(stream)
    torch.cuda.synchronize()
    t_plain = p0.elapsed_time(p1)
    clk = clocks.stop()
    del pl
    if pg:
        t_ms, t_plain = max_over_ranks([t_ms, t_plain], pg)
    value = G * args.steps * world / (t_ms / 1e3)
    plain = G * world / (t_plain / 1e3)
    # e2e: the host-buffer entry point on the first sub-batch, from pinned memory
    d0 = dgs[0]
    hs, hd, hw = (torch.from_numpy(x).pin_memory() for x in d0.to_host())
    packed = (hs.numpy(), hd.numpy(), hw.numpy(), d0.entry_off, d0.vertex_off)
    lv.run_batch(packed=packed)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        lv.run_batch(packed=packed)
    f1.record(stream)
    torch.cuda.synchronize()
    t_e2e = f0.elapsed_time(f1)
    e2e = d0.n_graphs * args.steps * world / (t_e2e / 1e3)
    del lv, ctxs
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        small = [p for p in params if p["n"] <= 5000][:256]
        t0 = time.perf_counter()
        for p in small:
            n, s_, d_, w_ = graphgen.sbm(p["n"], p["blocks"], p["p_in"], p["p_out"], 1, 4, seed=p["seed"] % (2 ** 62))
            O.Run(n, s_, d_, w_, n_threads=1)
        cpu_t = time.perf_counter() - t0
        cpu = {"value": len(small) / cpu_t, "unit": "graphs/s", "cores": 1, "kind": "port",
               "sample": f"{len(small)} graphs of the batched distribution with n <= 5000 (host SBM generator, "
                         f"generation included), one thread"}
    line = {
        "metric": "graphs/s batched vs plain at dQ<=1e-3", "value": value, "unit": "graphs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
        "config": {"workload": "batched SBMs", "graphs": G, "entries": E, "vertices": V,
                   "n_range": [64, 200000], "blocks": [4, 400], "avg_degree": [8, 32], "intra_fraction": 0.7,
                   "weights": "integer 1..4", "sub_batches": len(dgs), "batch_workers": nw, "seed": 3,
                   "inputs": "device-resident packed lists (device generator)",
                   "l2": "inputs larger than L2"},
        "tuning": tune,
        "plain": {"value": plain, "unit": "graphs/s", "ms_per_sweep": t_plain,
                  "speedup_batched_over_plain": value / plain,
                  "partitions_differing": mism, "max_abs_dq": dq_max},
        "roofline": None,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "graphs/s", "graphs": d0.n_graphs, "sample": "first sub-batch",
                "h2d_bytes_per_step": 12 * d0.n_entries + 12 * (d0.n_graphs + 1),
                "d2h_bytes_per_step": 4 * d0.n_vertices + 20 * d0.n_graphs},
        "clocks": clk,
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- serving form
def run_serving(args, world, rank, local, pg):
    """Poisson request stream served by the continuous-batching server
    (louvaingpu_b200.serving) against the plain per-request path on the same
    GPU, same arrival times: graphs/s and p50/p99/p99.9 latency."""
    import hashlib
    import torch
    from louvaingpu_b200 import Louvain, graphgen, kernel_launches
    from louvaingpu_b200.serving import Server
    torch.cuda.set_device(local)
    rng = np.random.default_rng(17 + rank)
    # request pool: SBMs of the batched distribution and R-MAT scale-22 giants
    params, groups = batched_plan(args.pool, 5 + rank, args.batch_entries)
    pool = [graphgen.sbm_batch_device(g, device=local) for g in groups]
    small = [(d, g) for d in pool for g in range(d.n_graphs)]
    giants = [graphgen.rmat_device(22, edge_factor=16, seed=100 + k, device=local) for k in range(args.giants)]
    torch.cuda.synchronize()
    R = args.requests
    is_giant = rng.random(R) < 0.02
    pick = rng.integers(0, 1 << 30, R)
    reqs = []
    for i in range(R):
        if is_giant[i] and giants:
            x = giants[pick[i] % len(giants)]
            reqs.append((x.src, x.dst, x.w, x.n_entries, x.n_vertices))
        else:
            d, g = small[pick[i] % len(small)]
            reqs.append(d.graph_ptrs(g))
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, R))
    free = torch.cuda.mem_get_info()[0]
    budget = int(min(150e9, free - 6e9))
    digest = lambda a: hashlib.blake2b(a.tobytes(), digest_size=8).hexdigest()  # noqa: E731

    # degree thresholds tuned once on a giant (the giants carry most of the
    # entries), outside the timed region; served and plain paths use the pair
    tune = {"tile_max_degree": 512, "block_max_degree": 4096, "autotuned": False}
    if not args.no_autotune and giants:
        with Louvain(device=local) as tl:
            x = giants[0]
            tl.load_edges_device(x.src, x.dst, x.w, x.n_entries, x.n_vertices)
            best, _ = tl.autotune(reps=2)
        tune = {"tile_max_degree": best[0], "block_max_degree": best[1], "autotuned": True,
                "tuned_on": "R-MAT scale-22 giant"}
    clocks = Clocks(local)
    clocks.start()
    # served: submit at the arrival times, results collected at the end
    with Server(n_slots=args.slots, hbm_budget=budget, max_batch_entries=int(args.batch_entries),
                tile_max_degree=tune["tile_max_degree"], block_max_degree=tune["block_max_degree"]) as srv:
        warm = [reqs[k] for k in range(min(64, R))]
        for s_, d_, w_, e_, n_ in warm:                       # warm-up requests (not timed)
            srv.submit(s_, d_, w_, e_, n_)
        srv.drain()
        srv.poll(1 << 20)
        l0 = kernel_launches()
        base = time.perf_counter()
        t_ref = None
        for i in range(R):
            wait = arrivals[i] - (time.perf_counter() - base)
            if wait > 0:
                time.sleep(wait)
            s_, d_, w_, e_, n_ = reqs[i]
            srv.submit(s_, d_, w_, e_, n_, part_out=np.empty(n_, np.int32), tag=i)
        srv.drain()
        wall = time.perf_counter() - base
        launches = kernel_launches() - l0
        out = srv.poll(R + 16)
        stats = srv.stats()
    out.sort(key=lambda r: r.tag)
    first = min(r.t_submit for r in out)
    served_lat = np.array([r.latency for r in out])
    served_span = max(r.t_done for r in out) - first
    served_digest = [digest(r.part) for r in out]
    served_q = np.array([r.q_final for r in out])
    bad_status = sum(1 for r in out if r.status != 0)
    # plain: one context, one request at a time, same arrival times
    pl = Louvain(device=local, tile_max_degree=tune["tile_max_degree"], block_max_degree=tune["block_max_degree"])
    torch.cuda.synchronize()
    plain_lat = np.zeros(R)
    mism, dq_max = 0, 0.0
    base = time.perf_counter()
    for i in range(R):
        wait = arrivals[i] - (time.perf_counter() - base)
        if wait > 0:
            time.sleep(wait)
        s_, d_, w_, e_, n_ = reqs[i]
        pl.load_edges_device(s_, d_, w_, e_, n_)
        res = pl.run()
        part = pl.partition()
        plain_lat[i] = (time.perf_counter() - base) - arrivals[i]
        if digest(part) != served_digest[i]:
            mism += 1
        dq_max = max(dq_max, abs(res.q_final - served_q[i]))
    plain_span = time.perf_counter() - base
    clk = clocks.stop()
    del pl
    if rank != 0:
        return
    pct = lambda a: {"p50_ms": float(np.percentile(a, 50) * 1e3), "p99_ms": float(np.percentile(a, 99) * 1e3),
                     "p999_ms": float(np.percentile(a, 99.9) * 1e3)}  # noqa: E731
    value = R * world / served_span
    line = {
        "metric": "graphs/s served (continuous batching) with p50/p99/p99.9 latency", "value": value,
        "unit": "graphs/s", "n_gpus": world, "steps": 1, "warmup": 1, "ms_per_step": served_span * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
        "config": {"workload": "Poisson request stream", "requests": R, "arrival_rate_per_s": args.rate,
                   "giant_fraction": 0.02, "giants": "R-MAT scale 22, edge factor 16, weights 1..16",
                   "giant_graphs_distinct": len(giants), "small": "SBMs of the batched distribution",
                   "small_pool_graphs": len(small), "hbm_budget_bytes": budget, "slots": args.slots,
                   "max_batch_entries": int(args.batch_entries), "l2": "inputs larger than L2"},
        "tuning": tune,
        "served": dict(pct(served_lat), graphs_per_s=value, span_s=served_span, batches=stats["batches"],
                       failed=bad_status, wall_s=wall),
        "plain": dict(pct(plain_lat), graphs_per_s=R / plain_span, span_s=plain_span),
        "speedup_served_over_plain": value / (R / plain_span),
        "same_alone_and_in_mix": {"partitions_differing": mism, "max_abs_dq": dq_max},
        "roofline": None, "cpu_baseline": None,
        "e2e": {"value": value, "unit": "graphs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(sum(r[4] for r in reqs) * 4),
                "note": "inputs device-resident (device generator); partitions returned to the host"},
        "clocks": clk, "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, pg)
        elif args.workload == "batched":
            run_batched(args, world, rank, local, pg)
        elif args.workload == "serving":
            run_serving(args, world, rank, local, pg)
        else:
            run_ours(args, world, rank, local, pg)
    finally:
        if pg:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
