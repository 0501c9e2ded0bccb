"""Move evaluation kernels (warp / block / hub degree bins) against the
oracle's restatement of the reference's decision (Module.cpp:1004-1123) on the
same snapshot."""
import numpy as np
import pytest

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu


def oracle_units(O, prep, st):
    return dict(out_off=prep.off, out_dst=prep.dst, out_f=st["f"], in_off=st["in_off"], in_src=st["in_src"],
                in_f=st["in_f"], p=st["p"], tw=prep.tw, dsize=st["dsize"], exit=st["exit"])


def compare(O, G, prep, st, part, allow_new=None):
    n = prep.n
    units = oracle_units(O, prep, st)
    ms = O.module_stats(n, st["p"], prep.tw, st["dsize"], prep.off, prep.dst, st["f"], part)
    se = float(ms["exit"][ms["count"] > 0].sum())
    bm_o, bd_o = O.evaluate(units, part, ms, se, allow_new)
    bm_g, bd_g = G.evaluate_moves(part, allow_new)
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


def test_degree_bins_hubs(built_lib, oracle_mod):
    """Units in every bin: degree <= 64 (warp), <= 2048 (block), hubs (global table)."""
    from relaxmap_b200 import Graph
    O = oracle_mod
    rng = np.random.default_rng(4)
    n = 6000
    src = [rng.integers(0, n, 40000)]
    dst = [rng.integers(0, n, 40000)]
    for hub, deg in ((0, 5000), (1, 3000), (2, 1500), (3, 100)):  # out-hubs and in-hubs
        src += [np.full(deg, hub), rng.integers(0, n, deg)]
        dst += [rng.integers(0, n, deg), np.full(deg, hub)]
    src = np.concatenate(src)
    dst = np.concatenate(dst)
    w = rng.uniform(1, 3, len(src))
    prep = O.prepare(O.from_edges(n, src, dst, w))
    st = O.initiate(prep)
    with Graph.from_edges(src, dst, w, n=n) as G:
        for k in (n, 40, 3):
            part = (rng.integers(0, k, n) * (n // k)).astype(np.int32)
            compare(O, G, prep, st, part)
