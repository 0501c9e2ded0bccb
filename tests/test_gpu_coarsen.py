"""Modules -> super-nodes: renumbering and super-node CSR/CSC bit-exact with
the reference given the same partition and the same edge flows."""
import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, golden

pytestmark = pytest.mark.gpu


def check_same(cv, ref):
    for k in ("out_off", "out_dst", "out_f", "in_off", "in_src", "in_f"):
        np.testing.assert_array_equal(cv[k], ref[k], err_msg=k)


@pytest.mark.parametrize("name", FIXTURES)
def test_against_reference(built_lib, oracle_mod, name):
    from relaxmap_b200 import Graph
    O = oracle_mod
    g = golden(name)
    part = g["part_seed1"]
    with Graph.from_file(GOLDEN / name) as G:
        f = G.initiate()["f"]
        off, dst, _, _ = G.links()
        cv = G.coarsen(part)
    assert cv["n_sn"] == len(g["sn_modidx"])
    np.testing.assert_array_equal(np.nonzero(cv["sn_of_mod"] >= 0)[0], g["sn_modidx"])
    # the oracle restatement on the GPU's own flows
    check_same(cv, O.convert(len(off) - 1, off, dst, f, part))
    # and the reference itself, fed the GPU's flows
    if O.reflib() is not None:
        R = O.Ref(path=GOLDEN / name)
        R.prepare(1)
        R.set_flows(f)
        R.set_partition(part)
        check_same(cv, R.convert())


@pytest.mark.parametrize("k", [2, 17, 400])
def test_random_partitions(built_lib, oracle_mod, k):
    from relaxmap_b200 import Graph, synth
    O = oracle_mod
    sg = synth.planted_partition(6000, 18, 400, 10, 300, 0.4, seed=11, weights="uniform")
    rng = np.random.default_rng(k)
    part = (rng.integers(0, k, sg.n) * 3).astype(np.int32)
    with Graph.from_edges(sg.src, sg.dst, sg.w, n=sg.n) as G:
        f = G.initiate()["f"]
        off, dst, _, _ = G.links()
        cv = G.coarsen(part)
    ref = O.convert(sg.n, off, dst, f, part)
    assert cv["n_sn"] == ref["n_sn"]
    np.testing.assert_array_equal(cv["sn_of_mod"], ref["sn_of_mod"])
    check_same(cv, ref)
