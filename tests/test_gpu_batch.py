"""Batched multi-graph x multi-attempt optimisation (rmx_batch_*).

Checked per graph against the single-graph path: the code length returned for
each graph is the code length of the returned partition computed from scratch
on that graph alone (1e-10 relative: fixed-point module sums against FP64),
which also checks the per-component flows of the disjoint union; a batch of
one graph and one attempt is exactly rmx_optimize; quality of the best of 4
attempts is within 0.5% of the single-graph optimiser."""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _graphs():
    from relaxmap_b200 import synth
    gs = []
    for k, spec in enumerate(synth.batched_graphs(6, seed=3, n_range=(200, 3000))):
        g = synth.batched_graph(spec)
        gs.append((g.n, g.src, g.dst, g.w))
    # a graph without links and one with dangling nodes and weights
    gs.append((5, np.zeros(0, np.int32), np.zeros(0, np.int32), None))
    rng = np.random.default_rng(0)
    s = rng.integers(0, 300, 2000).astype(np.int32)
    d = rng.integers(0, 300, 2000).astype(np.int32)
    keep = s % 7 != 0
    gs.append((300, s[keep], d[keep], rng.uniform(1, 5, keep.sum())))
    return gs


def _single_L(g, part):
    from relaxmap_b200 import Graph
    with Graph.from_edges(g[1], g[2], g[3], n=g[0]) as G:
        return G.codelength(part)


def _check_part(part, n, nm):
    assert len(part) == n
    assert part.min() == 0 and part.max() == nm - 1
    # first-appearance numbering
    first = []
    seen = set()
    for m in part.tolist():
        if m not in seen:
            seen.add(m)
            first.append(m)
    assert first == list(range(nm))


@pytest.mark.parametrize("waves", ["one", "many"])
def test_batch_matches_single_graph_code_lengths(built_lib, waves):
    from relaxmap_b200 import Batch
    gs = _graphs()
    with Batch(gs) as B:
        if waves == "many":
            B.set_wave(20_000, 10_000)
        r = B.optimize(seed=1, attempts=4)
        info = B.info()
    assert info["instances"] == 4 * len(gs)
    assert (info["waves"] > 1) == (waves == "many")
    for k, g in enumerate(gs):
        part = r["part"][k]
        _check_part(part, g[0], r["n_modules"][k])
        L = _single_L(g, part)
        assert abs(L - r["L"][k]) <= 1e-10 * abs(L), (k, L, r["L"][k])
        assert 0 <= r["best_attempt"][k] < 4


def test_batch_quality_against_single_optimiser(built_lib):
    from relaxmap_b200 import Batch, Graph
    gs = _graphs()[:6]
    with Batch(gs) as B:
        r = B.optimize(seed=1, attempts=4)
    for k, g in enumerate(gs):
        with Graph.from_edges(g[1], g[2], g[3], n=g[0]) as G:
            single = np.median([G.optimize(seed=s)["L"] for s in (1, 2, 3)])
        assert r["L"][k] <= 1.005 * single, (k, r["L"][k], single)


def test_batch_of_one_is_rmx_optimize(built_lib):
    from relaxmap_b200 import Batch, Graph, parse_file
    pf = parse_file(GOLDEN / "directNet_1k_sm_mu_03.txt")
    g = (pf["n"], pf["src"], pf["dst"], pf["w"])
    with Batch([g]) as B:
        r = B.optimize(seed=5, attempts=1)
    with Graph.from_edges(g[1], g[2], g[3], n=g[0]) as G:
        s = G.optimize(seed=5)
    assert r["L"][0] == s["L"]
    # same modules up to renumbering
    a, b = r["part"][0], np.asarray(s["part"])
    pairs = set(zip(a.tolist(), b.tolist()))
    assert len(pairs) == len(set(a.tolist())) == len(set(b.tolist()))


def test_batch_rejects_bad_input(built_lib):
    from relaxmap_b200 import Batch, RmxError
    with pytest.raises(RmxError):
        Batch([(3, np.array([0, 3], np.int32), np.array([1, 2], np.int32), None)])
    with pytest.raises(RmxError):
        Batch([(0, np.zeros(0, np.int32), np.zeros(0, np.int32), None)])


def test_batch_captured_loops_match_host_loops(built_lib, capfd):
    """A batch wave (a union of graph-attempt instances) runs its stage loops
    as captured while graphs from its first run; with per-sweep printing
    (verbose 2) the same loops are driven from the host. Same partitions, code
    lengths and best attempts."""
    from relaxmap_b200 import Batch
    gs = _graphs()
    with Batch(gs) as B:
        a = B.optimize(seed=2, attempts=3)
        b = B.optimize(seed=2, attempts=3, verbose=2)
    capfd.readouterr()  # the host loop's per-sweep lines
    np.testing.assert_array_equal(a["L"], b["L"])
    np.testing.assert_array_equal(a["best_attempt"], b["best_attempt"])
    for pa, pb in zip(a["part"], b["part"]):
        np.testing.assert_array_equal(pa, pb)
