"""Autotuner for the launch shape of move evaluation (rmx_set_tuning).

The grid cap of each degree bin (blocks per SM) and the degree bounds that
assign units to the bins change the time of an optimiser run, never its
result: every evaluation kernel loops over its bin's units by grid stride,
module statistics are exact integer sums, and every bin computes the same
change per candidate. The tuner
times full runs of a representative graph under candidate caps, one knob at a
time (coordinate descent, a few passes), keeps a candidate only when it is
faster by more than the noise margin, and checks that every candidate
reproduces the baseline code length bit for bit. A result is stored per device
(name and SM count) in a small JSON file; `load` applies it on the same kind
of device and ignores it elsewhere.

    python -m relaxmap_b200.autotune --nodes 200000 --out tuning.json
    python -m relaxmap_b200.autotune --graph net.txt --out tuning.json

and in a program: `relaxmap_b200.autotune.load("tuning.json")`.
"""
from __future__ import annotations

import argparse
import json
import statistics
from pathlib import Path
from typing import Callable

from ._lib import TUNING_FIELDS, get_tuning, set_tuning

# candidate grid caps (blocks per SM) of each bin and degree bounds of the
# bins (links); the defaults are among them, and every combination keeps
# warp <= mid <= block <= large
KNOBS: dict[str, tuple[int, ...]] = {
    "eval_mid_grid": (4, 6, 8, 12, 16),
    "eval_block_grid": (2, 3, 4, 6, 8),
    "eval_large_grid": (1, 2, 3),
    "eval_warp_grid": (2, 3, 4, 6, 8),
    "eval_reg_grid": (4, 6, 8, 12, 16),
    "warp_max_degree": (64, 96, 128),
    "mid_max_degree": (256, 384, 512),
    "block_max_degree": (768, 1024),
    "large_max_degree": (2048, 3072, 4096),
    "hub_partition_links": (512, 1024, 2048),
}
DEFAULTS = {"eval_mid_grid": 8, "eval_block_grid": 4, "eval_large_grid": 2, "eval_warp_grid": 3, "eval_reg_grid": 8,
            "warp_max_degree": 128, "mid_max_degree": 512, "block_max_degree": 1024, "large_max_degree": 4096,
            "hub_partition_links": 1024}
FORMAT = 1

# measure(setting) -> (milliseconds per run, code length of the run)
Measure = Callable[[dict], tuple[float, float]]


class TuningError(RuntimeError):
    pass


def tune(measure: Measure, knobs: dict[str, tuple[int, ...]] | None = None, start: dict | None = None,
         passes: int = 2, margin: float = 0.01) -> dict:
    """Coordinate descent over `knobs` from `start` (default: DEFAULTS).

    A candidate replaces the current setting when its time is below the best
    so far by more than `margin` (relative); a setting met again is not timed
    again. Every candidate must give the baseline code length exactly, else
    TuningError. Returns the setting, its time, the baseline time and the
    number of settings timed."""
    knobs = KNOBS if knobs is None else knobs
    cfg = dict(DEFAULTS if start is None else start)
    for k in knobs:
        if k not in TUNING_FIELDS:
            raise ValueError(f"unknown tuning field {k}")
    timed: dict[tuple, float] = {}  # each setting is timed once

    def run(c: dict) -> tuple[float, float]:
        key = tuple(sorted(c.items()))
        if key in timed:
            return timed[key], base_L
        ms, L = measure(dict(c))
        timed[key] = ms
        return ms, L

    base_L = None
    base_ms, base_L = run(cfg)
    best_ms = base_ms
    for _ in range(passes):
        changed = False
        for k, cands in knobs.items():
            for v in cands:
                if v == cfg[k]:
                    continue
                cand = dict(cfg, **{k: v})
                ms, L = run(cand)
                if L != base_L:
                    raise TuningError(f"{k}={v} changed the code length ({L!r} against {base_L!r}): "
                                      "the launch shape must not change results")
                if ms < best_ms * (1.0 - margin):
                    best_ms, cfg, changed = ms, cand, True
        if not changed:
            break
    return {"tuning": cfg, "ms": best_ms, "baseline_ms": base_ms, "timed_settings": len(timed)}


def device_key() -> str:
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name}|{p.multi_processor_count} SMs"


def gpu_measure(graph, seed: int = 1, reps: int = 3, **opts) -> Measure:
    """Times graph.optimize(seed=seed, **opts) with the flow recomputed each
    run, between CUDA events on the graph's stream, median of `reps` runs after
    one untimed run (which also captures the sweep graphs of a new setting)."""
    import torch
    stream = torch.cuda.ExternalStream(graph.stream_ptr())

    def measure(cfg: dict) -> tuple[float, float]:
        set_tuning(**cfg)
        graph.reset_flow()
        graph.optimize(seed=seed, **opts)
        times, L = [], None
        for _ in range(reps):
            graph.reset_flow()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = graph.optimize(seed=seed, **opts)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            if L is not None and r["L"] != L:
                raise TuningError("repeated runs of one setting gave different code lengths")
            L = r["L"]
        return statistics.median(times), L

    return measure


def tune_graph(graph, seed: int = 1, reps: int = 3, **kw) -> dict:
    """tune() on full optimiser runs of `graph`; the process keeps the setting
    it started with (the result is applied by `load` or set_tuning)."""
    before = get_tuning()
    try:
        res = tune(gpu_measure(graph, seed=seed, reps=reps), **kw)
    finally:
        set_tuning(**before)
    res["device"] = device_key()
    res["graph"] = {"nodes": graph.n, "links": graph.n_links}
    return res


def save(result: dict, path) -> None:
    out = {"format": FORMAT, "device": result["device"], "tuning": result["tuning"], "ms": result["ms"],
           "baseline_ms": result["baseline_ms"], "graph": result.get("graph")}
    Path(path).write_text(json.dumps(out, indent=1) + "\n")


def load(path, device: str | None = None) -> dict | None:
    """Apply a saved setting if it was tuned on this kind of device; returns
    the setting applied, or None (left unchanged) for another device."""
    d = json.loads(Path(path).read_text())
    if d.get("format") != FORMAT:
        raise ValueError(f"{path}: unknown tuning file format {d.get('format')!r}")
    if d["device"] != (device_key() if device is None else device):
        return None
    cfg = {k: int(v) for k, v in d["tuning"].items()}
    set_tuning(**cfg)
    return cfg


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--graph", help="edge list (.txt) or Pajek (.net) file to tune on")
    ap.add_argument("--nodes", type=int, default=200_000, help="synthetic planted-partition graph size")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--passes", type=int, default=2)
    ap.add_argument("--rmat", type=int, default=None,
                    help="tune on a synthetic R-MAT graph of this scale (edge factor 16, seed 42) instead")
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    from . import Graph, synth
    if a.graph:
        G = Graph.from_file(a.graph)
    elif a.rmat is not None:
        g = synth.rmat_device(a.rmat, 16, seed=42) if a.rmat >= 22 else synth.rmat(a.rmat, 16, seed=42)
        G = Graph.from_edges(g.src, g.dst, g.w, n=g.n)
    else:
        g = synth.config_mid(seed=42, n=a.nodes)
        G = Graph.from_edges(g.src, g.dst, g.w, n=g.n)
    with G:
        res = tune_graph(G, seed=a.seed, reps=a.reps, passes=a.passes)
    save(res, a.out)
    print(json.dumps(res))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
