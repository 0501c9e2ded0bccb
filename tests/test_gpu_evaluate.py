"""Move evaluation kernels (the register, warp, mid, block, large and hub
degree bins) against the oracle's restatement of the reference's decision
(Module.cpp:1004-1123, the same decision in prioritize_parallelMove
:1366-1485 and the super-node variants :2198-2313, :2555-2670) on the same
snapshot, at node level and at super-node level.

Bar: every unit's best change within 1e-11 x the largest change; its module
equal unless the oracle's change for the GPU's choice ties the best to 1e-12 x
that scale (exact ties resolve by FP64 rounding)."""
import numpy as np
import pytest

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu

# the engine's degree bins (out + in links of a unit at its level): upper bounds
BIN_MAX = {"reg8": 8, "reg16": 16, "reg32": 32, "warp": 128, "mid": 512, "block": 1024, "large": 4096,
           "hub": 1 << 62}


def bin_counts(deg):
    out, lo = {}, 0
    for name, hi in BIN_MAX.items():
        out[name] = int(((deg > lo) & (deg <= hi)).sum())
        lo = hi
    return out


def oracle_units(O, prep, st):
    return dict(out_off=prep.off, out_dst=prep.dst, out_f=st["f"], in_off=st["in_off"], in_src=st["in_src"],
                in_f=st["in_f"], p=st["p"], tw=prep.tw, dsize=st["dsize"], exit=st["exit"])


def check_units(O, units, part, bm_g, bd_g, allow_new=None):
    """The GPU's decisions (bm_g, bd_g) against the oracle's on units placed
    in modules part; returns how many units chose another module at a tie."""
    n_mod = max(len(part), int(part.max()) + 1)
    ms = O.module_stats(n_mod, units["p"], units["tw"], units["dsize"], units["out_off"], units["out_dst"],
                        units["out_f"], part)
    se = float(ms["exit"][ms["count"] > 0].sum())
    bm_o, bd_o = O.evaluate(units, part, ms, se, allow_new)
    scale = max(1.0, np.abs(bd_o).max())
    assert np.abs(bd_g - bd_o).max() <= 1e-11 * scale
    diff = np.nonzero(bm_g != bm_o)[0]
    for u in diff:  # only exact ties (to FP64 rounding) may resolve differently
        if bm_g[u] == -1 or bm_o[u] == -1:
            assert abs(bd_o[u]) <= 1e-12 * scale, (u, bm_g[u], bm_o[u], bd_o[u])
            continue
        d_g = O.delta_to(units, part, ms, se, int(u), int(bm_g[u]))
        assert abs(d_g - bd_o[u]) <= 1e-12 * scale, (u, bm_g[u], bm_o[u], d_g, bd_o[u])
    return len(diff)


def compare(O, G, prep, st, part, allow_new=None):
    units = oracle_units(O, prep, st)
    bm_g, bd_g = G.evaluate_moves(part, allow_new)
    return check_units(O, units, part, bm_g, bd_g, allow_new)


@pytest.mark.parametrize("name", ["flow.net", "directNet_1k_sm_mu_03.txt", "small_planted.txt"])
def test_fixture_partitions(built_lib, oracle_mod, name):
    from relaxmap_b200 import Graph
    O = oracle_mod
    prep = O.load(GOLDEN / name)
    st = O.initiate(prep)
    g = golden(name)
    n = prep.n
    rng = np.random.default_rng(0)
    with Graph.from_file(GOLDEN / name) as G:
        compare(O, G, prep, st, np.arange(n, dtype=np.int32))
        compare(O, G, prep, st, g["part_seed1"].astype(np.int32))
        part = (rng.integers(0, max(2, n // 20), n) * 7 % n).astype(np.int32)
        compare(O, G, prep, st, part)
        compare(O, G, prep, st, g["part_seed1"].astype(np.int32), np.ones(n, dtype=np.uint8))


def all_bins_graph(seed=4):
    """A sparse random graph plus groups of nodes whose out+in degree falls in
    each bin: at least 8 units per bin, hubs of 5000-6000 links included."""
    rng = np.random.default_rng(seed)
    n = 30000
    src = [rng.integers(0, n, n)]
    dst = [rng.integers(0, n, n)]
    hub = 0
    for deg, count in ((11, 16), (24, 16), (80, 16), (300, 12), (700, 10), (2500, 10), (5500, 8)):
        for _ in range(count):
            t = rng.choice(np.delete(np.arange(n), hub), deg, replace=False)
            k = deg // 2
            src += [np.full(k, hub), t[k:]]
            dst += [t[:k], np.full(deg - k, hub)]
            hub += 1
    src = np.concatenate(src)
    dst = np.concatenate(dst)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    return n, src, dst, rng.uniform(1, 3, len(src))


def test_degree_bins_all(built_lib, oracle_mod):
    """Node-level decisions with at least 8 units in every degree bin."""
    from relaxmap_b200 import Graph
    O = oracle_mod
    n, src, dst, w = all_bins_graph()
    prep = O.prepare(O.from_edges(n, src, dst, w))
    st = O.initiate(prep)
    deg = np.diff(prep.off) + np.diff(st["in_off"])
    occ = bin_counts(deg)
    assert min(occ.values()) >= 8, occ
    rng = np.random.default_rng(5)
    with Graph.from_edges(src, dst, w, n=n) as G:
        for k in (n, 40, 3):
            part = (rng.integers(0, k, n) * (n // k)).astype(np.int32)
            compare(O, G, prep, st, part)
        compare(O, G, prep, st, np.arange(n, dtype=np.int32), np.ones(n, dtype=np.uint8))


@pytest.mark.parametrize("tuning", [
    {"large_max_degree": 1024, "hub_partition_links": 64},
    {"large_max_degree": 32, "block_max_degree": 32, "mid_max_degree": 32, "warp_max_degree": 32,
     "hub_partition_links": 1 << 30},
])
def test_hub_partitions(built_lib, oracle_mod, tuning):
    """The hub pipeline under other partition sizes: partitions of 64 links
    (many per unit), and one partition per unit for every unit above 32 links,
    so that units of 2500 and 5500 distinct neighbour modules overfill the
    partition table and are aggregated in rounds."""
    from relaxmap_b200 import Graph, get_tuning, set_tuning
    O = oracle_mod
    n, src, dst, w = all_bins_graph()
    prep = O.prepare(O.from_edges(n, src, dst, w))
    st = O.initiate(prep)
    before = get_tuning()
    rng = np.random.default_rng(6)
    try:
        set_tuning(**tuning)
        with Graph.from_edges(src, dst, w, n=n) as G:
            compare(O, G, prep, st, np.arange(n, dtype=np.int32))
            for k in (400, 3):
                part = (rng.integers(0, k, n) * (n // k)).astype(np.int32)
                compare(O, G, prep, st, part)
    finally:
        set_tuning(**before)


# ------------------------------------------------------------ super-node level

def sn_units(O, G, part):
    """The first super-node level of part as the reference forms it
    (convertModulesToSuperNodes: super-node CSR/CSC with FP64 link sums; each
    super-node's flow, teleport weight, dangling flow and exit are its
    module's, SuperNode(Module, int) Node.cpp:76-106)."""
    st = G.initiate()
    off, dst, _, tw = G.links()
    f = st["f"]
    ref = O.convert(len(off) - 1, off, dst, f, part)
    mods = np.unique(part)
    grp = np.searchsorted(mods, part)
    dsize = np.where(st["dangling"] != 0, st["p"], 0.0)
    ms = O.module_stats(len(mods), st["p"], tw, dsize, off, dst, f, grp)
    units = dict(out_off=ref["out_off"], out_dst=ref["out_dst"], out_f=ref["out_f"], in_off=ref["in_off"],
                 in_src=ref["in_src"], in_f=ref["in_f"], p=ms["P"], tw=ms["TW"], dsize=ms["D"], exit=ms["exit"])
    return units, mods, grp


def compare_sn(O, G, part, sn_part, allow_new=None):
    units, mods, _ = sn_units(O, G, part)
    sn_part = np.ascontiguousarray(sn_part, dtype=np.int32)
    bm_g, bd_g = G.evaluate_sn_moves(part, sn_part, allow_new)
    check_units(O, units, sn_part, bm_g, bd_g, allow_new)
    return np.diff(units["out_off"]) + np.diff(units["in_off"])


@pytest.mark.parametrize("name", ["directNet_1k_sm_mu_03.txt", "small_planted.txt"])
def test_supernode_level_from_run(built_lib, oracle_mod, name):
    """Super-node levels of a real run: the reference's own first superstep
    (one-thread node sweeps, seed 1) gives the super-nodes; they are evaluated
    as singletons (the start of the super-node stage), grouped as the
    reference's final partition groups their first members, and randomly."""
    from relaxmap_b200 import Graph
    O = oracle_mod
    prep = O.load(GOLDEN / name)
    st = O.initiate(prep)
    _, part1, _ = O.node_sweeps(prep, st, 1, True, 0.0, 1e-3, 10)
    part1 = part1.astype(np.int32)
    final = golden(name)["part_seed1"].astype(np.int32)
    rng = np.random.default_rng(1)
    with Graph.from_file(GOLDEN / name) as G:
        mods = np.unique(part1)
        ns = len(mods)
        assert ns > 4
        first = np.array([np.nonzero(part1 == m)[0][0] for m in mods])
        compare_sn(O, G, part1, mods)
        compare_sn(O, G, part1, final[first])
        compare_sn(O, G, part1, mods[rng.integers(0, max(2, ns // 4), ns)])
        compare_sn(O, G, part1, mods, np.ones(ns, dtype=np.uint8))


@pytest.mark.parametrize("k,k2", [(17, 5), (60, 12), (400, 40), (1500, 100)])
def test_supernode_level_bins(built_lib, oracle_mod, k, k2):
    """Super-node levels whose units fall in the register, warp, mid and block
    bins (random partitions of a 6000-node planted-partition graph into k
    modules, the super-nodes grouped into k2 modules)."""
    from relaxmap_b200 import Graph, synth
    O = oracle_mod
    sg = synth.planted_partition(6000, 18, 400, 10, 300, 0.4, seed=11, weights="uniform")
    rng = np.random.default_rng(k)
    part = (rng.integers(0, k, sg.n) * 3).astype(np.int32)
    with Graph.from_edges(sg.src, sg.dst, sg.w, n=sg.n) as G:
        mods = np.unique(part)
        ns = len(mods)
        deg = compare_sn(O, G, part, mods)
        compare_sn(O, G, part, mods[rng.integers(0, k2, ns)])
    assert deg.max() > 0
