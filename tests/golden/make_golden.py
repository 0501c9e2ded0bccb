"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run where the reference sources exist (RMX_REFERENCE_DIR, else the oracle
recipe's REF_DIR in oracle/Makefile); it builds oracle/_ref/ from them.

    python tests/golden/make_golden.py

Writes, per fixture graph <g>:
  <g> (input copy)         flow.net, flow.txt, directNet_1k_sm_mu_03.txt from the
                           reference's data/, small_planted.txt from the seeded
                           generator (1000 nodes, the small benchmark shape)
  <g>.ref.npz              from the reference compiled from its own sources:
                             loader output (summed edge map), node weights
                             initiate at 1 thread: p, f (CSR order), singleton
                             exit, dangling, L0, sum p log p, iterations
                             8 seeds x {1, 8} threads, prior: final code length
                             (incremental and recomputed, bits), module count
                             the seed-1 one-thread partition and its coarsening
                             (convertModulesToSuperNodes) on the reference flows
  flow.ref.tree / flow.ref.clu   the reference CLI's output files for flow.net
                                 (seed 1, 1 thread, 1e-3, 0.0, 10, prior)
  quality.ref.npz          larger seeded graphs regenerated by the tests
                           (QUALITY_CASES): the reference's final code length
                           (bits, recomputed) for seeds 1..8 at 8 threads, prior

    python tests/golden/make_golden.py quality [case ...]   # only quality.ref.npz
"""
from __future__ import annotations

import shutil
import subprocess
import sys
import tarfile
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from relaxmap_b200 import synth  # noqa: E402

REF = O.REF_SRC
SEEDS = list(range(1, 9))


def copy_inputs():
    shutil.copy(REF / "data" / "flow.net", HERE / "flow.net")
    shutil.copy(REF / "data" / "flow.txt", HERE / "flow.txt")
    with tarfile.open(REF / "data" / "directNet_1k_sm_mu_network.tgz") as t:
        m = t.getmember("directNet_1k_sm_mu_03.txt")
        data = t.extractfile(m).read()
    (HERE / "directNet_1k_sm_mu_03.txt").write_bytes(data)
    synth.config_small(seed=42).write_edge_list(HERE / "small_planted.txt")


def golden(name: str):
    path = HERE / name
    out = {}
    R = O.Ref(path=path)
    s, d, w = R.map_edges()
    out.update(map_src=s, map_dst=d, map_w=w, node_w=R.node_weights(), n=np.int64(R.n))
    R.prepare(1)
    off, dst, f = R.links()
    nd = R.nodes()
    out.update(off=off, dst=dst, f=f, p=nd["p"], tw=nd["tw"], exit=nd["exit"], dangling=nd["dangling"],
               L0=np.float64(R.codelength()), all_log_all=np.float64(R.R.rmxref_all_log_all(R._h)))
    g = O.load(path)
    st = O.initiate(g)
    out["iters"] = np.int64(st["iters"])
    Lb, Lc, nm = [], [], []
    for threads in (1, 8):
        for seed in SEEDS:
            Rk = O.Ref(path=path)
            Rk.prepare(threads)
            r = Rk.partition(seed=seed, threads=threads, threshold=1e-3, vthresh=0.0, max_iter=10, prior=True)
            Lb.append(r["L_bits"])
            Lc.append(r["L_computed_bits"])
            nm.append(r["n_modules"])
            if threads == 1 and seed == 1:
                out["part_seed1"] = r["part"]
    out.update(final_L_bits=np.array(Lb).reshape(2, -1), final_L_computed_bits=np.array(Lc).reshape(2, -1),
               final_n_modules=np.array(nm).reshape(2, -1), seeds=np.array(SEEDS), threads=np.array([1, 8]))
    R.set_partition(out["part_seed1"])
    out["part_seed1_codelength"] = np.float64(R.calc_codelength())
    cv = R.convert()
    for k in ("modidx", "out_off", "out_dst", "out_f", "in_off", "in_src", "in_f"):
        out["sn_" + k] = cv[k]
    np.savez_compressed(HERE / (name + ".ref.npz"), **out)
    print(name, "N", R.n, "links", len(dst), "median L bits (1 thr)", np.median(out["final_L_bits"][0]),
          "(8 thr)", np.median(out["final_L_bits"][1]))


# name -> generator call; the tests rebuild the same graphs from these seeds
QUALITY_CASES = {
    "rmat14": lambda: synth.rmat(14, 16, seed=42),
    "planted20k_mid": lambda: synth.config_mid(seed=42, n=20_000),
    "planted20k_adjoint": lambda: synth.config_adjoint(seed=42, n=20_000),
    # the bench's CPU sample of the R-MAT family, and the full 1M-node mid graph
    "rmat18": lambda: synth.rmat(18, 16, seed=42),
    "planted1m_mid": lambda: synth.config_mid(seed=42, n=1_000_000),
}


def quality(names=None):
    """The reference's 8-seed final code lengths of QUALITY_CASES (all, or the
    named ones, merged into the existing file)."""
    out = {}
    qf = HERE / "quality.ref.npz"
    if names and qf.exists():
        with np.load(qf) as z:
            out = {k: z[k] for k in z.files}
    for name, make in QUALITY_CASES.items():
        if names and name not in names:
            continue
        g = make()
        ld = O.from_edges(g.n, g.src, g.dst, g.w)
        Lc = []
        for seed in SEEDS:
            R = O.Ref(loaded=ld)
            R.prepare(8)
            Lc.append(R.partition(seed=seed, threads=8, threshold=1e-3, vthresh=0.0, max_iter=10,
                                  prior=True)["L_computed_bits"])
        out[name] = np.array(Lc)
        print(name, "N", g.n, "E", g.m, "median L bits", np.median(Lc), flush=True)
        np.savez_compressed(qf, **out)


def cli_outputs():
    with tempfile.TemporaryDirectory() as td:
        src = Path(td) / "in"
        src.mkdir()
        shutil.copy(HERE / "flow.net", src / "flow.net")
        subprocess.run([str(O.REF_BIN), "1", str(src / "flow.net"), "1", "1", "1e-3", "0.0", "10", td, "prior"],
                       check=True, capture_output=True)
        shutil.copy(Path(td) / "flow.tree", HERE / "flow.ref.tree")
        shutil.copy(Path(td) / "flow.clu", HERE / "flow.ref.clu")


if __name__ == "__main__":
    O.build(reference=True)
    if sys.argv[1:2] == ["quality"]:
        quality(sys.argv[2:])
        sys.exit(0)
    copy_inputs()
    for name in ("flow.net", "flow.txt", "directNet_1k_sm_mu_03.txt", "small_planted.txt"):
        golden(name)
    cli_outputs()
    quality()
