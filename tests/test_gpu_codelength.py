"""From-scratch FP64 code length (calculateCodeLength) on the GPU."""
import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", FIXTURES)
def test_reference_partition(built_lib, name):
    from relaxmap_b200 import Graph
    g = golden(name)
    with Graph.from_file(GOLDEN / name) as G:
        L = G.codelength(g["part_seed1"])
        L0 = G.initiate()["L0"]
        Ls = G.codelength(np.arange(G.n, dtype=np.int32))
    assert abs(L - float(g["part_seed1_codelength"])) <= 1e-10
    assert abs(Ls - L0) <= 1e-10


def test_random_partitions_vs_oracle(built_lib, oracle_mod):
    from relaxmap_b200 import Graph, synth
    O = oracle_mod
    sg = synth.planted_partition(4000, 15, 200, 10, 100, 0.3, seed=9, weights="uniform")
    prep = O.prepare(O.from_edges(sg.n, sg.src, sg.dst, sg.w))
    st = O.initiate(prep)
    rng = np.random.default_rng(1)
    with Graph.from_edges(sg.src, sg.dst, sg.w, n=sg.n) as G:
        for k in (1, 7, 300, sg.n):
            part = rng.integers(0, k, sg.n).astype(np.int32) * (sg.n // k)
            assert abs(G.codelength(part) - O.codelength(prep, st, part)) <= 1e-10
        part = sg.community
        assert abs(G.codelength(part) - O.codelength(prep, st, part)) <= 1e-10
