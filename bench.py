"""Benchmark: edges/s per full optimiser run on one B200 (or N replicas).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload rmat24|mid|small|rmat<scale>|batched|adjoint]

Default workload: R-MAT scale 24 (16,777,216 nodes, edge factor 16,
(0.57, 0.19, 0.19, 0.05), self-loops and duplicates removed, unweighted),
drawn on the GPU from seed 42; the largest configuration that fits one B200.

One step = one full run of the map-equation optimiser (flow power iteration,
all supersteps, final partition) on the workload graph:
  value  graph resident in HBM (CSR/CSC built once, outside the timed region),
         device time of K runs (CUDA events on the engine's stream); each run
         recomputes the flow; edges/s = input links / time per run
  e2e    the same through the C ABI from pinned HOST buffers every step:
         rmx_graph_create (host->device copy, device CSR/CSC build),
         rmx_optimize (partition copied back), rmx_graph_destroy
The single-graph optimiser does not shard: with N GPUs every rank runs its own
replica (no collective); value = all ranks' links / the slowest rank's time.
--impl reference times the reference (compiled from its own sources, all host
threads) on a bounded sample of the same workload family (R-MAT scale 18 for
the R-MAT workloads, 200,000 nodes for mid): not the same graph as ours.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "edges/s per full run"
UNIT = "edges/s"


def workload(name: str, nodes: int | None = None):
    from relaxmap_b200 import synth
    if name == "small":
        g = synth.config_small(seed=42)
        desc = "planted partition N=1000, out-degree power law 2 (mean 20, max 50), communities [10,50], mu=0.3, unweighted"
    elif name == "mid":
        n = nodes or 1_000_000
        g = synth.config_mid(seed=42, n=n)
        desc = (f"planted partition N={n:,}, out-degree power law 2 (mean 20, max 1000), communities power law "
                "[20,1000], mu=0.4, weights U[1,10]")
    elif name.startswith("rmat"):
        scale = int(name[4:])
        if scale >= 22:  # drawn on the GPU: the host generator takes minutes at this size
            g = synth.rmat_device(scale, 16, seed=42)
            gen = "torch CUDA generator, seed 42"
        else:
            g = synth.rmat(scale, 16, seed=42)
            gen = "numpy generator, seed 42"
        desc = (f"R-MAT scale {scale}, edge factor 16, (0.57,0.19,0.19,0.05), self-loops/duplicates removed, "
                f"unweighted ({gen})")
    else:
        raise SystemExit(f"unknown workload {name}")
    return g, desc


def reference_sample(name: str):
    """The bounded CPU sample of the workload family (the reference's
    std::map build and OpenMP sweeps take hours on the full R-MAT scale-24
    graph and minutes on the 1M-node mid graph): R-MAT scale 18 with the same
    parameters, or the mid distributions at 200,000 nodes."""
    from relaxmap_b200 import synth
    if name == "mid":
        g = synth.config_mid(seed=42, n=200_000)
        return g, "planted partition N=200,000 with the mid distributions (1/5 of the nodes)"
    if name == "small":
        return synth.config_small(seed=42), "the full small graph"
    g = synth.rmat(18, 16, seed=42)
    return g, "R-MAT scale 18, edge factor 16, (0.57,0.19,0.19,0.05), self-loops/duplicates removed (numpy, seed 42)"


# The reference's 8-seed final code lengths (bits) committed by
# tests/golden/make_golden.py: the full mid graph, and the R-MAT family's CPU sample.
QUALITY_GOLDEN = ROOT / "tests" / "golden" / "quality.ref.npz"


def reference_quality(case: str):
    import numpy as np
    if not QUALITY_GOLDEN.exists():
        return None
    with np.load(QUALITY_GOLDEN) as z:
        return [float(x) for x in z[case]] if case in z.files else None


def sample_quality(G_cls, sg, case: str, seeds: int = 8) -> dict | None:
    """Our median code length over seeds 1..8 on a graph the reference was run
    on 8 times (its golden median), and the relative gap."""
    ref = reference_quality(case)
    if ref is None:
        return None
    with G_cls.from_edges(sg.src, sg.dst, sg.w, n=sg.n) as G:
        ours = [G.optimize(seed=k)["L_bits"] for k in range(1, seeds + 1)]
    rm = statistics.median(ref)
    om = statistics.median(ours)
    return {"ref_median_bits": rm, "gpu_median_bits": om, "gap": (om - rm) / rm, "seeds": seeds}


def run_reference(g, threads: int, seed: int = 1) -> dict:
    """Reference optimiser on graph g: its loader-equivalent edge map, edge
    preparation, initiate and partition (the 'w/o file IO' region)."""
    import numpy as np

    from oracle import oracle as O
    ld = O.Loaded(g.n, [], np.ones(g.n), float(g.n), g.src.astype(np.int64), g.dst.astype(np.int64),
                  np.ones(g.m) if g.w is None else g.w)
    R = O.Ref(loaded=ld)
    tp = R.prepare(threads)
    r = R.partition(seed=seed, threads=threads, threshold=1e-3, vthresh=0.0, max_iter=10, prior=True)
    return dict(seconds=tp + r["seconds"], L_bits=r["L_computed_bits"], n_modules=r["n_modules"])


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for k, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(k)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def write_edge_list(path, g, chunk: int = 1_000_000) -> int:
    """g as an edge-list file, 'src dst w' per line with weights to 6
    significant digits (the format the drop-in loader reads); returns its size
    in bytes."""
    with open(path, "w") as f:
        for s in range(0, g.m, chunk):
            a, b = g.src[s:s + chunk].tolist(), g.dst[s:s + chunk].tolist()
            if g.w is None:
                f.write("".join(f"{x} {y}\n" for x, y in zip(a, b)))
            else:
                f.write("".join(f"{x} {y} {z:.6g}\n" for x, y, z in zip(a, b, g.w[s:s + chunk].tolist())))
    return os.path.getsize(path)


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# DRAM bytes (read + write) per link evaluated by the dominant evaluation
# kernel, keyed by (workload, degree bin): one ncu capture of that kernel (one
# launch, dram__bytes_read.sum + dram__bytes_write.sum, a single pass) in the
# evaluation snapshot of the benched graph (--eval-snapshot: every node against
# singleton modules), divided by the links that launch read; the command and
# the counters are in profiles/eval_large_rmat24.md.
EVAL_TRAFFIC_PER_LINK = {("rmat24", "large"): (9.31e9 + 6.87e6) / 97_860_671}

DOMINANT_BIN = "large"

# The kernel (or kernel chain) each degree bin of the evaluation launches.
EVAL_BIN_KERNELS = {"reg": "k_eval_reg", "warp": "k_eval_warp", "mid": "k_eval_block<128, 1024>",
                    "block": "k_eval_block<256, 2048>", "large": "k_eval_block<512, 8192>",
                    "hub": "k_hub_plan/links/offsets/eval/finish/mark"}


def profile_run(g, desc: str):
    """One graph build, flow and optimiser run: the unit that ncu launch lists
    and kernel captures are taken over."""
    from relaxmap_b200 import Graph
    G = Graph.from_edges(g.src, g.dst, g.w, n=g.n)
    G.initiate()
    G.set_profiling(True)
    t0 = time.perf_counter()
    r = G.optimize(seed=1)
    dt = time.perf_counter() - t0
    p = G.profile()
    G.close()
    print(json.dumps({"workload": desc, "nodes": g.n, "links": g.m, "seconds": dt, "L_bits": r["L_bits"],
                      "n_modules": r["n_modules"], "profile": p}))


def eval_bytes(links: int, units: int, cands: int, modules: int) -> float:
    """Compulsory bytes of one evaluation launch group: 16 per link read (id,
    fixed-point flow, neighbour's module), 40 per unit (module id, statistics,
    proposal), 40 per module statistics record read (at most one per candidate)."""
    return 16.0 * links + 40.0 * units + 40.0 * min(cands, modules)


def eval_snapshot(g, desc: str):
    """One launch group of the evaluation kernels: every node evaluated against
    singleton modules (rmx_evaluate_moves)."""
    import numpy as np

    from relaxmap_b200 import Graph
    G = Graph.from_edges(g.src, g.dst, g.w, n=g.n)
    G.initiate()
    p0 = G.profile()
    G.evaluate_moves(np.arange(g.n, dtype=np.int32))
    p1 = G.profile()
    G.close()
    d = {k: p1[k] - p0[k] for k in ("links_evaluated", "units_evaluated", "candidates_evaluated")}
    d["bytes"] = eval_bytes(d["links_evaluated"], d["units_evaluated"], d["candidates_evaluated"], g.n)
    d["bin_links"] = {b: p1["eval_bins"][b]["links"] - p0["eval_bins"][b]["links"] for b in p1["eval_bins"]}
    print(json.dumps({"workload": desc, "nodes": g.n, "links": g.m, "eval_group": d}))


def slowest_over_ranks(vals, pg, device):
    """Element-wise max over ranks: the slowest rank sets the job's time.
    Every rank makes this call at the same point (one all_reduce)."""
    import torch
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    if pg is not None:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def job_throughput(world: int, units_per_rank: float, seconds: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return world * units_per_rank / seconds


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat24")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--with-io", action="store_true",
                    help="also time the drop-in path with file IO: edge-list file -> load (all host cores) -> "
                         "optimise -> .tree/.clu (one GPU; the input file is written first, untimed)")
    ap.add_argument("--nodes", type=int, default=None, help="mid workload: node count (smaller profiling cases)")
    ap.add_argument("--graphs", type=int, default=4096, help="batched workload: number of graphs")
    ap.add_argument("--profile-run", action="store_true",
                    help="build the graph, then exactly one optimiser run (seed 1); prints the engine counters "
                         "(the command profiled by ncu)")
    ap.add_argument("--eval-snapshot", action="store_true",
                    help="build the graph, then one move evaluation of every node against singleton modules (one "
                         "launch group of the evaluation kernels); prints its counters and compulsory bytes (the "
                         "command whose DRAM traffic ncu measures for the roofline)")
    args = ap.parse_args()
    world, rank, local = dist_setup()

    if args.impl == "reference":
        if rank != 0:
            return
        bench_reference(args, world)
        return

    import numpy as np
    import torch

    from relaxmap_b200 import Graph, get_tuning

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist

    if args.workload == "batched":
        bench_batched(args, world, rank, pg)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    if args.workload == "adjoint":
        bench_adjoint(args, world, rank, pg)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    g, desc = workload(args.workload, args.nodes)
    E = g.m
    if args.profile_run:
        profile_run(g, desc)
        return
    if args.eval_snapshot:
        eval_snapshot(g, desc)
        return
    # ---- resident graph
    G = Graph.from_edges(g.src, g.dst, g.w, n=g.n)
    G.initiate()
    stream = torch.cuda.ExternalStream(G.stream_ptr())
    for _ in range(args.warmup):
        G.optimize(seed=1)
    # timed without the library's per-kernel timing events (their presence
    # switches the sweeps from CUDA graphs to direct launches)
    launches0 = G.profile()["kernel_launches"]
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    results = []
    with Clocks(torch.cuda.current_device()) as clk:
        e0.record(stream)
        for k in range(args.steps):
            G.reset_flow()  # every step recomputes the flow, as the reference's timed region does
            results.append(G.optimize(seed=1 + k))
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    gpu_launches = G.profile()["kernel_launches"] - launches0
    # one more run with the timing events: kernel-class times and bytes for the roofline
    G.set_profiling(True)
    G.reset_flow()
    G.optimize(seed=1)
    prof = G.profile()
    G.set_profiling(False)
    ms_step = ms / args.steps
    ms_step_max = slowest_over_ranks([ms_step], pg, "cuda")[0]
    value = job_throughput(world, E, ms_step_max / 1e3)
    L_bits = [r["L_bits"] for r in results]

    # ---- end to end through the C ABI with pinned host buffers
    src = torch.from_numpy(g.src).pin_memory()
    dst = torch.from_numpy(g.dst).pin_memory()
    w = torch.from_numpy(g.w).pin_memory() if g.w is not None else None
    e2e_steps = max(1, min(args.steps, 3))
    Gw = Graph.from_host_ptrs(src.data_ptr(), dst.data_ptr(), w.data_ptr() if w is not None else 0, E, g.n)
    Gw.optimize(seed=1)
    Gw.close()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    build_s = opt_s = close_s = dev_s = 0.0
    for k in range(e2e_steps):
        tb = time.perf_counter()
        Ge = Graph.from_host_ptrs(src.data_ptr(), dst.data_ptr(), w.data_ptr() if w is not None else 0, E, g.n)
        to = time.perf_counter()
        build_s += to - tb
        Ge.optimize(seed=1 + k)  # the partition is copied back to host memory inside
        tc = time.perf_counter()
        opt_s += tc - to
        dev_s += Ge.profile()["total_ms"] / 1e3  # device time of that run (flow + supersteps)
        Ge.close()
        close_s += time.perf_counter() - tc
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    build_s /= e2e_steps
    opt_s /= e2e_steps
    close_s /= e2e_steps
    dev_s /= e2e_steps
    e2e_value = job_throughput(world, E, slowest_over_ranks([e2e_s], pg, "cuda")[0])

    # ---- with file IO, as the reference's command line runs: file in, .tree/.clu out
    with_io = None
    if args.with_io and world == 1:
        import tempfile
        with tempfile.TemporaryDirectory(prefix=".bench_io_", dir=ROOT) as td:
            path = os.path.join(td, "graph.txt")
            size = write_edge_list(path, g)
            io_steps = max(1, min(args.steps, 2))
            t0 = time.perf_counter()
            for k in range(io_steps):
                Gf = Graph.from_file(path)
                rf = Gf.optimize(seed=1 + k)
                Gf.write_outputs(rf["part"], rf["L"], td, "/graph")
                Gf.close()
            io_s = (time.perf_counter() - t0) / io_steps
        with_io = {"value": E / io_s, "unit": UNIT, "seconds_per_step": io_s, "input_bytes": size,
                   "path": "edge-list file -> rmx_graph_load_file (all host cores) -> rmx_optimize -> "
                           "rmx_write_outputs (.tree/.clu)", "note": "weights written to 6 significant digits"}

    # ---- code length against the reference's 8-seed median: the same graph
    # (mid), or, where the reference cannot run the full graph, its CPU sample
    quality = {"L_bits_median": statistics.median(L_bits), "n_modules": results[0]["n_modules"],
               "seeds": len(L_bits)}
    sg_q, rdesc = reference_sample(args.workload)
    if args.workload == "mid" and (args.nodes or 1_000_000) == 1_000_000:
        ref = reference_quality("planted1m_mid")
        if ref is not None:
            rm = statistics.median(ref)
            quality.update(ref_median_bits=rm, gap=(quality["L_bits_median"] - rm) / rm)
    elif args.workload.startswith("rmat") and rank == 0:
        quality["on_reference_sample"] = sample_quality(Graph, sg_q, "rmat18")
        quality["note"] = ("the reference cannot run the full graph within a run's time (hours on the host): its "
                           "8-seed median is compared on the CPU sample, R-MAT scale 18")

    # ---- roofline of the dominant kernel: the large bin's k_eval_block<512, 8192>,
    # the top kernel of the launch list on R-MAT scale 24 (the bins run
    # concurrently, so their stream timers overlap and cannot rank them). Its
    # time is its own stream's events around each launch (other bins run
    # beside it), its compulsory bytes come from its own links, units and
    # candidates.
    pk = peaks()
    ev = prof["eval"]
    bins = prof["eval_bins"]
    dom = DOMINANT_BIN if bins[DOMINANT_BIN]["launches"] > 0 else max(bins, key=lambda b: bins[b]["ms"])
    db = bins[dom]
    achieved = db["bytes"] / (db["ms"] / 1e3) / 1e9 if db["ms"] > 0 else 0.0
    per_link = EVAL_TRAFFIC_PER_LINK.get((args.workload, dom))
    traffic = None
    if per_link is not None and db["launches"] > 0:
        traffic = per_link * db["links"] / db["launches"]
    group_gbs = ev["bytes"] / (ev["ms"] / 1e3) / 1e9 if ev["ms"] > 0 else 0.0
    shares = {k: prof[k]["ms"] for k in ("spmv", "eval", "commit", "coarsen", "codelen", "other")}
    tot = sum(shares.values()) or 1.0

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, seed 42)",
        "config": {"workload": desc, "nodes": g.n, "links": E, "solver": "seed 1..K, threshold 1e-3, vThresh 0.0, "
                   "maxIter 10, prior", "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": f"inputs larger than L2 (resident graph ~{(E * 104 + g.n * 420) / 1e9:.1f} GB)",
                   "timed_region": "value: the flow (power iteration, edge flows) and every superstep on the "
                                   "resident graph; the device CSR/CSC build (part of the reference's w/o-IO "
                                   "region, OmpRelaxmap.cpp:103-162) is outside it and inside e2e",
                   "reference_arm": {"same_config": False, "sample": rdesc},
                   "launch_tuning": get_tuning()},
        "quality": quality,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(E * (8 + (8 if w is not None else 0))),
                "d2h_bytes_per_step": int(4 * g.n + 8),
                "split_ms": {"graph_create": build_s * 1e3, "optimize_wall": opt_s * 1e3,
                             "optimize_device": dev_s * 1e3, "graph_destroy": close_s * 1e3},
                "note": "a fresh handle per step: graph_create copies the host arrays in and builds the CSR/CSC; "
                        "optimize_wall includes the flow, the run and the partition copied back"},
        "roofline": {"kernel": f"move evaluation, {dom} bin ({EVAL_BIN_KERNELS[dom]})", "bound": "hbm",
                     "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                     "peak_source": pk["source"], "traffic": traffic,
                     "traffic_note": "per launch: DRAM bytes per link from one ncu capture of this kernel on this "
                                     "graph x the links per launch here; the random gathers (the neighbour's module, "
                                     "the candidate's statistics and terms) each move a 32-byte sector",
                     "traffic_frac": (traffic / (db["ms"] / max(db["launches"], 1) / 1e3) / 1e9 / pk["hbm_gbs"]
                                      if traffic is not None and db["ms"] > 0 else None),
                     "algorithmic_bytes_per_launch": db["bytes"] / max(db["launches"], 1),
                     "launch_ms_avg": db["ms"] / max(db["launches"], 1),
                     "bins": {b: {"ms": round(v["ms"], 3), "launches": v["launches"], "links": v["links"],
                                  "GB/s": round(v["bytes"] / v["ms"] / 1e6, 1) if v["ms"] > 0 else None}
                              for b, v in bins.items()},
                     "launch_group": {"GB/s": group_gbs, "frac": group_gbs / pk["hbm_gbs"],
                                      "bytes_per_launch": ev["bytes"] / max(ev["launches"], 1),
                                      "ms_avg": ev["ms"] / max(ev["launches"], 1),
                                      "note": "one sub-batch: every bin, concurrently on six streams"}},
        "kernel_time_share": {k: round(v / tot, 4) for k, v in shares.items()},
        "profiled_run": {"level_ms": prof["level_ms"],
                         "eval_bin_ms": {b: round(v["ms"], 3) for b, v in prof["eval_bins"].items()},
                         "links_evaluated": prof["links_evaluated"], "units_evaluated": prof["units_evaluated"],
                         "candidates_evaluated": prof["candidates_evaluated"], "sweeps": prof["sweeps"],
                         "power_iters": prof["power_iters"]},
        "gpu_launches": int(gpu_launches),
        "clocks": clk.summary(),
    }
    if with_io is not None:
        line["with_io"] = with_io
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            sg, sdesc = sg_q, rdesc
            r = run_reference(sg, os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": sg.m / r["seconds"], "unit": UNIT, "cores": os.cpu_count(),
                                    "kind": "reference", "sample": sdesc + f" ({sg.m} links, {r['seconds']:.2f} s, "
                                    f"L={r['L_bits']:.5f} bits)"}
        except Exception as e:  # the reference build is test infrastructure; report, do not fail
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    if rank == 0:
        print(json.dumps(line))
    G.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


BATCH_ATTEMPTS = 16
BATCH_METRIC = "graphs/s (16 attempts per graph)"


def _gen_batched(spec):
    from relaxmap_b200 import synth
    g = synth.batched_graph(spec)
    return (g.n, g.src, g.dst, g.w)


def bench_batched(args, world: int, rank: int, pg):
    """The batched workload: --graphs graphs (N ~ U[200,20000], mu ~ U[0.1,0.6],
    mean degree ~ U[5,30]), each optimised 16 times (best kept). Graphs are
    sharded over the ranks by estimated links (LPT); one step = every rank's
    share through rmx_batch_optimize."""
    import multiprocessing

    import numpy as np
    import torch

    from relaxmap_b200 import Batch, get_tuning, synth
    from relaxmap_b200.sharding import combine, lpt_assign
    G = args.graphs
    specs = synth.batched_graphs(G, seed=42)
    mine = lpt_assign([s[0] * s[1] for s in specs], world)[rank]
    with multiprocessing.get_context("spawn").Pool(min(os.cpu_count() or 1, 32)) as pool:
        gs = pool.map(_gen_batched, [specs[i] for i in mine.tolist()], chunksize=8)
    links = int(sum(len(g[1]) for g in gs))
    nodes = int(sum(g[0] for g in gs))
    with Batch(gs[:min(8, len(gs))]) as W:
        for _ in range(args.warmup):
            W.optimize(seed=1, attempts=BATCH_ATTEMPTS)
    B = Batch(gs)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    dev_s, wall_s = 0.0, 0.0
    with Clocks(torch.cuda.current_device()) as clk:
        for k in range(args.steps):
            t0 = time.perf_counter()
            r = B.optimize(seed=1 + k, attempts=BATCH_ATTEMPTS)
            wall_s += time.perf_counter() - t0
            dev_s += B.info()["device_ms"] / 1e3
    info = B.info()
    B.close()
    dev_max, wall_max = slowest_over_ranks([dev_s / args.steps, wall_s / args.steps], pg, "cuda")
    L_bits = combine(G, mine, r["L_bits"], pg, "cuda")
    n_mod = combine(G, mine, r["n_modules"], pg, "cuda")
    line = {
        "metric": BATCH_METRIC, "value": G / dev_max, "unit": "graphs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_max * 1e3, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, seed 42)",
        "config": {"workload": f"{G} planted-partition graphs, N~U[200,20000], mu~U[0.1,0.6], mean out-degree "
                               "~U[5,30] (power law 2, max 10x mean), communities [10,200]; 16 attempts each",
                   "graphs": G, "rank0_graphs": len(mine), "rank0_nodes": nodes, "rank0_links": links,
                   "rank0_waves": info["waves"], "rank0_instances": info["instances"],
                   "parallelism": f"graphs sharded over {world} ranks (LPT by links)" if world > 1 else "single GPU",
                   "timing": "value: device time of the optimiser runs (graphs resident); e2e: wall time of "
                             "rmx_batch_optimize from host arrays (packing, copies, CSR build, runs)",
                   "launch_tuning": get_tuning()},
        "quality": {"L_bits_mean": float(np.mean(L_bits)), "n_modules_mean": float(np.mean(n_mod))},
        "e2e": {"value": G / wall_max, "unit": "graphs/s", "h2d_bytes_per_step": int(links * 16),
                "d2h_bytes_per_step": int(nodes * 4 + len(mine) * 16)},
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1:
        # the same graphs one by one through rmx_optimize (16 attempts each): a
        # sample of every 64th graph of this rank, device time per graph
        from relaxmap_b200 import Graph
        sample = gs[::64]
        seq_s = 0.0
        for g in sample:
            with Graph.from_edges(g[1], g[2], g[3], n=g[0]) as Gs:
                Gs.optimize(seed=1, attempts=BATCH_ATTEMPTS)
                seq_s += Gs.profile()["total_ms"] / 1e3
        seq_rate = len(sample) / seq_s
        line["sequential_plain_gpu"] = {"value": seq_rate, "unit": "graphs/s", "sample": f"every 64th graph "
                                        f"({len(sample)} graphs), rmx_optimize with 16 attempts each, device time",
                                        "batched_over_sequential": line["value"] / seq_rate}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        secs = []
        for g in gs[:4]:
            sg = synth.SynthGraph(g[0], g[1], g[2], g[3])
            secs.append(run_reference(sg, os.cpu_count() or 1)["seconds"])
        per_graph = BATCH_ATTEMPTS * float(np.mean(secs))
        line["cpu_baseline"] = {"value": 1.0 / per_graph, "unit": "graphs/s", "cores": os.cpu_count(),
                                "kind": "reference",
                                "sample": f"the reference on the first 4 graphs of the batch, one attempt each "
                                          f"({', '.join(f'{x:.2f}' for x in secs)} s), x16 attempts"}
    if rank == 0:
        print(json.dumps(line))


ADJ_METRIC = "edges/s per gradient (forward + backward)"


def bench_adjoint(args, world: int, rank: int, pg):
    """The adjoint workload: dL/dw and dL/dtau of the code length of a fixed
    partition (the planted communities) on N=1e6, mean degree 20, mu=0.3,
    lognormal weights. One step = rmx_adjoint_backward: the stationary flow
    recomputed, module terms, the transposed solve, dL/dw for every link
    returned to host memory."""
    import numpy as np
    import torch

    from relaxmap_b200 import Graph, synth
    n = args.nodes or 1_000_000
    g = synth.config_adjoint(seed=42, n=n)
    desc = (f"planted partition N={n:,}, out-degree power law 2 (mean 20, max 1000), communities power law "
            "[20,1000], mu=0.3, weights lognormal(0,1); fixed partition = planted communities")
    E = g.m
    part = np.ascontiguousarray(g.community, dtype=np.int32)
    G = Graph.from_edges(g.src, g.dst, g.w, n=g.n)
    G.initiate()
    stream = torch.cuda.ExternalStream(G.stream_ptr())
    # the gradient lands in pinned host memory (the caller's choice of buffer)
    grad_host = torch.empty(max(G.n_links, 1), dtype=torch.float64).pin_memory().numpy()
    for _ in range(args.warmup):
        G.adjoint_backward(part, out=grad_host)
    G.set_profiling(True)
    launches0 = G.profile()["kernel_launches"]
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(torch.cuda.current_device()) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            r = G.adjoint_backward(part, out=grad_host)
        e1.record(stream)
        torch.cuda.synchronize()
    ms_step = e0.elapsed_time(e1) / args.steps
    prof = G.profile()
    G.set_profiling(False)
    # the forward pass alone (flow + code length of the partition): median over
    # calls, each between its own events on the engine's stream
    fwd = []
    for _ in range(max(args.steps, 3)):
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        G.adjoint_forward(part)
        f1.record(stream)
        torch.cuda.synchronize()
        fwd.append(f0.elapsed_time(f1))
    fwd_ms = statistics.median(fwd)
    ms_max = slowest_over_ranks([ms_step], pg, "cuda")[0]
    value = job_throughput(world, E, ms_max / 1e3)
    # end to end: graph built from pinned host buffers, gradient back in host memory
    src = torch.from_numpy(g.src).pin_memory()
    dst = torch.from_numpy(g.dst).pin_memory()
    w = torch.from_numpy(g.w).pin_memory()
    # one untimed handle first, as in the default workload's end-to-end loop
    Gw = Graph.from_host_ptrs(src.data_ptr(), dst.data_ptr(), w.data_ptr(), E, g.n)
    Gw.adjoint_backward(part, out=grad_host)
    Gw.close()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e2e_steps = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        Ge = Graph.from_host_ptrs(src.data_ptr(), dst.data_ptr(), w.data_ptr(), E, g.n)
        Ge.adjoint_backward(part, out=grad_host)
        Ge.close()
    e2e_s = slowest_over_ranks([(time.perf_counter() - t0) / e2e_steps], pg, "cuda")[0]
    pk = peaks()
    ad = prof["adjoint"]
    achieved = ad["bytes"] / (ad["ms"] / 1e3) / 1e9 if ad["ms"] > 0 else 0.0
    line = {
        "metric": ADJ_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, seed 42)",
        "config": {"workload": desc, "nodes": g.n, "links": E, "tau": 0.15,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (resident graph ~1.5 GB)"},
        "quality": {"L_nats": r["L"], "dL_dtau": r["dL_dtau"]},
        "forward_ms": fwd_ms, "backward_over_forward": ms_step / fwd_ms,
        "e2e": {"value": job_throughput(world, E, e2e_s), "unit": UNIT, "h2d_bytes_per_step": int(E * 16),
                "d2h_bytes_per_step": int(G.n_links * 8 + 16)},
        "roofline": {"kernel": "transposed flow solve (k_adj_solve)", "bound": "hbm", "achieved": achieved,
                     "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                     "peak_source": pk["source"], "traffic": None,
                     "algorithmic_bytes_per_launch": ad["bytes"] / max(ad["launches"], 1),
                     "launch_ms_avg": ad["ms"] / max(ad["launches"], 1),
                     "solve_sweeps_per_launch": prof["adjoint_iters"] / max(ad["launches"], 1)},
        "gpu_launches": int(prof["kernel_launches"] - launches0),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import adjoint as AD
        from oracle import oracle as O
        sg = synth.config_adjoint(seed=42, n=100_000)
        ld = O.from_edges(sg.n, sg.src, sg.dst, sg.w)
        pr = O.prepare(ld)
        t0 = time.perf_counter()
        AD.backward(pr.off, pr.dst, pr.w, pr.tw, np.asarray(sg.community))
        secs = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": sg.m / secs, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"CPU FP64 adjoint (numpy/scipy) on the same shape at N=100,000 "
                                          f"({sg.m} links, {secs:.2f} s); the reference has no gradient"}
    if rank == 0:
        print(json.dumps(line))
    G.close()


def bench_reference(args, world):
    sg, sdesc = reference_sample(args.workload)
    threads = os.cpu_count() or 1
    try:
        for _ in range(args.warmup):
            run_reference(sg, threads)
        secs = []
        for k in range(args.steps):
            secs.append(run_reference(sg, threads, seed=1 + k)["seconds"])
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference harness failed: {e}"}))
        return
    s = sum(secs) / len(secs)
    v = sg.m / s
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, seed 42)",
        "config": {"workload": sdesc, "nodes": sg.n, "links": sg.m, "solver": "seed 1..K, threshold 1e-3, "
                   "vThresh 0.0, maxIter 10, prior", "parallelism": f"{threads} host threads",
                   "same_config": False,
                   "note": f"a bounded CPU sample of the {args.workload} workload family (the full graph takes "
                           "hours on the host); timed over the reference's w/o-IO region: edge preparation, "
                           "initiate and every superstep"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sdesc},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


if __name__ == "__main__":
    main()
