"""The optimiser's own coarsening (convert_to_supernodes: hash aggregation of
fixed-point link flows, aggregate_links) against the reference's
convertModulesToSuperNodes (Module.cpp:3008-3077) on the same partition and
the same edge flows.

Bars:
* super-node numbering (ascending module id, Module.cpp:3015-3022) and the
  CSR/CSC structure are bit-exact once each engine row is ordered by its
  other end (the engine keeps rows in hash order; the reference's rows come
  sorted by destination from a std::map, its in-links by source);
* every fixed-point link sum equals the exact integer sum of the per-link
  fixed-point flows rint(f * 2^62) of its member links, and the super-node
  statistics (flow, teleport weight, dangling flow, out-flow) equal the
  exact integer sums of their members';
* converted to FP64, a link sum of k member links lies within
  k * 2^-62 + (k + 1) * 2^-52 * |ref| of the reference's FP64 sum (the
  fixed-point rounding of each term plus the reference's own FP64 rounding).
Groups of more than 16384 member links take the split pipeline (links
partitioned by destination over many blocks); the two-group, second-level
(300, 2) and huge-group cases cover it. The second-level case converts the super-nodes again (the super-node stage's
repeated conversion, OmpRelaxmap.cpp:379-411): the engine aggregates the first
level's links, the reference converts the composite node partition."""
import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, golden

pytestmark = pytest.mark.gpu

FX = 2.0 ** 62


def to_fx(x):
    return np.rint(np.asarray(x) * FX).astype(np.int64)


def rows_sorted(off, idx, *vals):
    row = np.repeat(np.arange(len(off) - 1), np.diff(off))
    o = np.lexsort((idx, row))
    return (idx[o],) + tuple(v[o] for v in vals)


def expected_links(off, dst, f, grp, nsn):
    """Crossing links grouped by (source group, destination group): the
    exact fixed-point sums and the number of member links of each pair, in
    CSR order and in CSC order."""
    src = np.repeat(np.arange(len(off) - 1), np.diff(off))
    a, b = grp[src].astype(np.int64), grp[dst].astype(np.int64)
    c = a != b
    q = to_fx(f[c])
    out = {}
    for name, key in (("csr", a[c] * nsn + b[c]), ("csc", b[c] * nsn + a[c])):
        uk, inv = np.unique(key, return_inverse=True)
        s = np.zeros(len(uk), dtype=np.int64)
        np.add.at(s, inv, q)
        out[name] = (s, np.bincount(inv, minlength=len(uk)))
    return out


def check_against(cv, ref, off, dst, f, p, tw, dangling, grp):
    nsn = cv["n_sn"]
    assert nsn == ref["n_sn"]
    np.testing.assert_array_equal(cv["out_off"], ref["out_off"])
    np.testing.assert_array_equal(cv["in_off"], ref["in_off"])
    od, ofx = rows_sorted(cv["out_off"], cv["out_dst"], cv["out_fx"])
    isrc, ifx = rows_sorted(cv["in_off"], cv["in_src"], cv["in_fx"])
    np.testing.assert_array_equal(od, ref["out_dst"])
    np.testing.assert_array_equal(isrc, ref["in_src"])
    exp = expected_links(off, dst, f, grp, nsn)
    np.testing.assert_array_equal(ofx, exp["csr"][0])
    np.testing.assert_array_equal(ifx, exp["csc"][0])
    for got, rf, cnt in ((ofx, ref["out_f"], exp["csr"][1]), (ifx, ref["in_f"], exp["csc"][1])):
        tol = cnt * 2.0 ** -62 + (cnt + 1) * 2.0 ** -52 * np.abs(rf)
        assert np.all(np.abs(got / FX - rf) <= tol)
    # super-node statistics: exact member sums, and the reference's FP64 values
    st = cv["sn_stat"]
    P = np.zeros(nsn, dtype=np.int64)
    np.add.at(P, grp, to_fx(p))
    TW = np.zeros(nsn, dtype=np.int64)
    np.add.at(TW, grp, to_fx(tw))
    D = np.zeros(nsn, dtype=np.int64)
    np.add.at(D, grp[dangling != 0], to_fx(p[dangling != 0]))
    OUT = np.zeros(nsn, dtype=np.int64)
    np.add.at(OUT, np.repeat(np.arange(nsn), np.diff(cv["out_off"])), ofx)
    np.testing.assert_array_equal(st[:, 0], P)
    np.testing.assert_array_equal(st[:, 1], TW)
    np.testing.assert_array_equal(st[:, 2], D)
    np.testing.assert_array_equal(st[:, 3], OUT)
    # against the reference's FP64 values: its node flows are its own (only the
    # edge flows were handed to it), which agree with the device's to 1e-12
    # relative L1 (test_gpu_flow); elementwise 1e-13 relative covers them
    cnt = np.bincount(grp, minlength=nsn)
    for k, name in ((0, "size"), (1, "tw"), (2, "dsize")):
        tol = cnt * 2.0 ** -62 + ((cnt + 1) * 2.0 ** -52 + 1e-13) * np.abs(ref[name])
        assert np.all(np.abs(st[:, k] / FX - ref[name]) <= tol), name
    # the exit flow from those statistics: every term is non-negative, so the
    # reference's own rounding is at most (members + crossing links + a few
    # operations) x 2^-52 of the exit, plus the fixed-point rounding of each
    # term and the node-flow difference above
    Pd, TWd, Dd, OUTd = (st[:, k] / FX for k in range(4))
    ex = 0.15 * (1.0 - TWd) * Pd + 0.85 * (OUTd + (1.0 - TWd) * Dd)
    nlinks = np.zeros(nsn, dtype=np.int64)  # member links leaving the super-node
    src_sn = grp[np.repeat(np.arange(len(off) - 1), np.diff(off))]
    np.add.at(nlinks, src_sn[src_sn != grp[dst]], 1)
    tol = ((cnt + nlinks + 8) * 2.0 ** -52 + 1e-13) * np.maximum(np.abs(ref["exit"]), Pd) + (cnt + nlinks) * 2.0 ** -62
    assert np.all(np.abs(ex - ref["exit"]) <= tol)


def reference_level(O, G, part, path=None, graph=None):
    st = G.initiate()
    off, dst, _, tw = G.links()
    f = st["f"]
    if O.reflib() is not None:
        if path is not None:
            R = O.Ref(path=path)
        else:
            R = O.Ref(loaded=O.from_edges(graph.n, graph.src, graph.dst, graph.w))
        R.prepare(1)
        R.set_flows(f)
        R.set_partition(part)
        ref = R.convert()
        np.testing.assert_array_equal(ref["modidx"], np.unique(part))
    else:  # the oracle restatement (bit-exact to the reference on the structure and FP64 sums)
        ref = O.convert(len(off) - 1, off, dst, f, part)
        ref["modidx"] = np.unique(part)
        nsn = ref["n_sn"]
        grp = np.searchsorted(ref["modidx"], part)
        ms = O.module_stats(nsn, st["p"], tw, np.where(st["dangling"] != 0, st["p"], 0.0), off, dst, f, grp)
        ref.update(size=ms["P"], tw=ms["TW"], dsize=ms["D"], exit=ms["exit"])
    grp = np.searchsorted(ref["modidx"], part).astype(np.int64)
    return ref, off, dst, f, st["p"], tw, st["dangling"], grp


@pytest.mark.parametrize("name", FIXTURES)
def test_fixtures(built_lib, oracle_mod, name):
    from relaxmap_b200 import Graph
    part = golden(name)["part_seed1"].astype(np.int32)
    with Graph.from_file(GOLDEN / name) as G:
        ref, off, dst, f, p, tw, dg, grp = reference_level(oracle_mod, G, part, path=GOLDEN / name)
        cv = G.coarsen_engine(part)
    np.testing.assert_array_equal(np.nonzero(cv["sn_of_mod"] >= 0)[0], ref["modidx"])
    check_against(cv, ref, off, dst, f, p, tw, dg, grp)


@pytest.fixture(scope="module")
def planted():
    from relaxmap_b200 import synth
    return synth.planted_partition(6000, 18, 400, 10, 300, 0.4, seed=11, weights="uniform")


@pytest.mark.parametrize("k", [2, 17, 400, 6000])
def test_random_partitions(built_lib, oracle_mod, planted, k):
    from relaxmap_b200 import Graph
    sg = planted
    rng = np.random.default_rng(k)
    part = (rng.integers(0, k, sg.n) * (sg.n // k)).astype(np.int32)
    with Graph.from_edges(sg.src, sg.dst, sg.w, n=sg.n) as G:
        ref, off, dst, f, p, tw, dg, grp = reference_level(oracle_mod, G, part, graph=sg)
        cv = G.coarsen_engine(part)
    check_against(cv, ref, off, dst, f, p, tw, dg, grp)


@pytest.mark.parametrize("part_links", [64, 1024, 1 << 30])
def test_huge_groups(built_lib, oracle_mod, planted, part_links):
    """A group of half the nodes (about 49,000 member links, above the bound
    past which a group's links are summed by the split pipeline) next to
    singletons, under three partition sizes of that pipeline: many small
    partitions; the default; and one partition holding all of the group's
    3000 distinct destinations, more than half its table, so that it is
    summed in subsets."""
    from relaxmap_b200 import Graph, get_tuning, set_tuning
    sg = planted
    part = np.arange(sg.n, dtype=np.int32)
    part[: sg.n // 2] = 0
    before = get_tuning()
    try:
        set_tuning(hub_partition_links=part_links)
        with Graph.from_edges(sg.src, sg.dst, sg.w, n=sg.n) as G:
            ref, off, dst, f, p, tw, dg, grp = reference_level(oracle_mod, G, part, graph=sg)
            cv = G.coarsen_engine(part)
    finally:
        set_tuning(**before)
    assert np.diff(cv["out_off"])[0] > 2048  # the group's row: distinct destinations
    check_against(cv, ref, off, dst, f, p, tw, dg, grp)


def test_large_level():
    """A level of more than 2^22 links over 5000 groups (long rows packed in
    chunks by many blocks): the CSR sums equal the exact integer sums of the
    member links, and the CSC is exactly the transpose of the CSR."""
    from relaxmap_b200 import Graph, synth
    sg = synth.planted_partition(400_000, 14, 400, 10, 300, 0.5, seed=5)
    rng = np.random.default_rng(8)
    part = (rng.integers(0, 5000, sg.n) * 7).astype(np.int32)
    with Graph.from_edges(sg.src, sg.dst, sg.w, n=sg.n) as G:
        st = G.initiate()
        off, dst, _, _ = G.links()
        cv = G.coarsen_engine(part)
    nsn = cv["n_sn"]
    grp = np.searchsorted(np.unique(part), part).astype(np.int64)
    exp = expected_links(off, dst, st["f"], grp, nsn)
    assert len(exp["csr"][0]) > (1 << 22) and nsn > 2048
    od, ofx = rows_sorted(cv["out_off"], cv["out_dst"], cv["out_fx"])
    np.testing.assert_array_equal(ofx, exp["csr"][0])
    # the CSC as (column, row, flow) triples equals the CSR's, ordered the same way
    orow = np.repeat(np.arange(nsn), np.diff(cv["out_off"]))
    icol = np.repeat(np.arange(nsn), np.diff(cv["in_off"]))
    a = np.lexsort((orow, cv["out_dst"]))
    b = np.lexsort((cv["in_src"], icol))
    np.testing.assert_array_equal(cv["out_dst"][a], icol[b])
    np.testing.assert_array_equal(orow[a], cv["in_src"][b])
    np.testing.assert_array_equal(cv["out_fx"][a], cv["in_fx"][b])


@pytest.mark.parametrize("k1,k2", [(400, 17), (1500, 300), (300, 2)])
def test_second_level(built_lib, oracle_mod, planted, k1, k2):
    """Super-nodes converted again: level 2 aggregated from level 1's links
    equals the reference's conversion of the composite node partition."""
    from relaxmap_b200 import Graph
    sg = planted
    rng = np.random.default_rng(k1 + k2)
    part = (rng.integers(0, k1, sg.n) * 3).astype(np.int32)
    part2 = np.arange(sg.n, dtype=np.int32)  # identity for unused ids
    mods = np.unique(part)
    part2[mods] = rng.choice(mods, k2, replace=False)[rng.integers(0, k2, len(mods))]
    comp = part2[part]
    with Graph.from_edges(sg.src, sg.dst, sg.w, n=sg.n) as G:
        ref, off, dst, f, p, tw, dg, grp = reference_level(oracle_mod, G, comp, graph=sg)
        cv = G.coarsen_engine(part, part2)
    np.testing.assert_array_equal(np.nonzero(cv["sn_of_mod"] >= 0)[0], ref["modidx"])
    check_against(cv, ref, off, dst, f, p, tw, dg, grp)


def test_second_level_fixture(built_lib, oracle_mod):
    """The same on the reference's 1000-node network with its seed-1 modules
    merged pairwise."""
    from relaxmap_b200 import Graph
    name = "directNet_1k_sm_mu_03.txt"
    part = golden(name)["part_seed1"].astype(np.int32)
    mods = np.unique(part)
    part2 = np.arange(len(part), dtype=np.int32)
    part2[mods] = mods[(np.arange(len(mods)) // 2) * 2]
    comp = part2[part]
    with Graph.from_file(GOLDEN / name) as G:
        ref, off, dst, f, p, tw, dg, grp = reference_level(oracle_mod, G, comp, path=GOLDEN / name)
        cv = G.coarsen_engine(part, part2)
    check_against(cv, ref, off, dst, f, p, tw, dg, grp)
