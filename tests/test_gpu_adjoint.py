"""rmx_adjoint_forward / rmx_adjoint_backward against the CPU FP64 adjoint
(oracle/adjoint.py, itself pinned against centred differences of the
reference's code length).

Tolerances: the device solves both systems by iteration to a relative L1
change of 1e-15, the oracle by sparse LU; L agrees to 1e-12 relative, the flow
to 1e-12 relative L1, dL/dw to 1e-9 relative L1 (and 1e-9 of the largest
component elementwise), dL/dtau to 1e-9 relative."""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

O = pytest.importorskip("oracle.oracle")
AD = pytest.importorskip("oracle.adjoint")


def _rel_l1(a, b):
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


def _check(G, part, tau):
    off, dst, w, tw = G.links()
    ref = AD.backward(off, dst, w, tw, part, t=tau)
    fw = G.adjoint_forward(part, tau, want_p=True)
    assert abs(fw["L"] - ref["L"]) <= 1e-12 * abs(ref["L"])
    assert _rel_l1(fw["p"], ref["p"]) <= 1e-12
    bw = G.adjoint_backward(part, tau)
    assert abs(bw["L"] - ref["L"]) <= 1e-12 * abs(ref["L"])
    g, rg = bw["dL_dw"], ref["dL_dw"]
    assert len(g) == len(rg)
    assert _rel_l1(g, rg) <= 1e-9, _rel_l1(g, rg)
    assert np.abs(g - rg).max() <= 1e-9 * np.abs(rg).max()
    assert abs(bw["dL_dtau"] - ref["dL_dt"]) <= 1e-9 * abs(ref["dL_dt"])
    return bw


@pytest.mark.parametrize("name", ["directNet_1k_sm_mu_03.txt", "flow.net", "small_planted.txt"])
@pytest.mark.parametrize("tau", [0.15, 0.3])
def test_adjoint_golden(built_lib, name, tau):
    from relaxmap_b200 import Graph
    with Graph.from_file(GOLDEN / name) as G:
        part = G.optimize(seed=1)["part"]
        if tau == 0.15:  # at the reference's teleportation the forward is calculateCodeLength
            assert abs(G.adjoint_forward(part, tau)["L"] - G.codelength(part)) <= 1e-12 * G.codelength(part)
        _check(G, part, tau)


def test_adjoint_planted_lognormal(built_lib):
    """The adjoint workload's shape (lognormal weights, mu = 0.3) at 20K nodes,
    with dangling nodes and a partition that is not an optimum."""
    from relaxmap_b200 import Graph, synth
    g = synth.planted_partition(20_000, 20, 1000, 20, 1000, 0.3, seed=5, weights="lognormal")
    src, dst, w = g.src, g.dst, g.w
    keep = src % 97 != 0  # some nodes without out-links
    with Graph.from_edges(src[keep], dst[keep], w[keep], n=g.n) as G:
        part = np.asarray(G.optimize(seed=2)["part"], dtype=np.int32)
        rng = np.random.default_rng(3)
        moved = rng.random(g.n) < 0.05
        part[moved] = rng.integers(0, g.n, moved.sum())
        _check(G, part, 0.15)


def test_adjoint_rejects_bad_input(built_lib):
    from relaxmap_b200 import Graph, RmxError
    with Graph.from_file(GOLDEN / "flow.net") as G:
        part = np.zeros(G.n, dtype=np.int32)
        for tau in (0.0, 1.0, -0.5):
            with pytest.raises(RmxError) as e:
                G.adjoint_forward(part, tau)
            assert e.value.status == 1
        bad = part.copy()
        bad[0] = G.n
        with pytest.raises(RmxError):
            G.adjoint_backward(bad, 0.15)


def test_adjoint_solve_cap_reports_no_convergence(built_lib):
    """A ring where every node links to the next (weight 1) and the one after
    (weight 0.5) mixes slowly: |lambda_2| of its walk is 1 - O((2 pi / n)^2),
    so the solve's error falls by barely (1 - tau) per sweep. At tau = 1e-4 the
    1e-15 tolerance is out of reach of the 4000-sweep cap and the call reports
    RMX_ERR_NO_CONVERGENCE instead of an inaccurate gradient. The handle stays
    usable: at tau = 0.15 the same graph converges (~180 sweeps) and matches
    the oracle (two out-links per node, so dL/dw is not identically zero)."""
    from relaxmap_b200 import Graph, RmxError
    n = 1000
    a = np.arange(n, dtype=np.int32)
    src = np.concatenate([a, a])
    dst = np.concatenate([(a + 1) % n, (a + 2) % n]).astype(np.int32)
    w = np.concatenate([np.ones(n), np.full(n, 0.5)])
    part = np.repeat(np.arange(3, dtype=np.int32), [100, 200, 700])
    with Graph.from_edges(src, dst, w, n=n) as G:
        with pytest.raises(RmxError) as e:
            G.adjoint_backward(part, 1e-4)
        assert e.value.status == 6  # RMX_ERR_NO_CONVERGENCE
        _check(G, part, 0.15)


def test_adjoint_full_size_config(built_lib):
    """The adjoint workload at full size: N = 1,000,000, mean out-degree 20,
    mu = 0.3, lognormal(0, 1) weights, the planted communities as the fixed
    partition.

    * Against the CPU FP64 adjoint (Neumann-series solves to 1e-16): dL/dw
      within 1e-6 relative L1 and 1e-6 of the largest component, dL/dtau
      within 1e-6 relative, L within 1e-12 relative.
    * Against centred differences of rmx_adjoint_forward (h = 1e-6 of the
      link's weight; the graph rebuilt from its own CSR with one weight
      moved): 64 links, 32 drawn at random and the 32 of largest |dL/dw|.
      A difference quotient carries the forward's own rounding, about
      1e-14 |L| per evaluation (the flow solve stops at a relative L1 change
      of 1e-15), divided by 2h: the bar is 1e-6 |g| plus that floor."""
    from relaxmap_b200 import Graph, synth
    g = synth.config_adjoint(seed=42, n=1_000_000)
    part = np.ascontiguousarray(g.community, dtype=np.int32)
    with Graph.from_edges(g.src, g.dst, g.w, n=g.n) as G:
        off, dst, w, tw = G.links()
        bw = G.adjoint_backward(part)
    ref = AD.backward(off, dst, w, tw, part)
    grad, rg = bw["dL_dw"], ref["dL_dw"]
    assert abs(bw["L"] - ref["L"]) <= 1e-12 * abs(ref["L"])
    assert _rel_l1(grad, rg) <= 1e-6, _rel_l1(grad, rg)
    assert np.abs(grad - rg).max() <= 1e-6 * np.abs(rg).max()
    assert abs(bw["dL_dtau"] - ref["dL_dt"]) <= 1e-6 * abs(ref["dL_dt"])
    # centred differences on links of the prepared graph (CSR order = gradient order)
    src = np.repeat(np.arange(g.n, dtype=np.int32), np.diff(off))
    rng = np.random.default_rng(11)
    pick = np.unique(np.concatenate([rng.choice(len(w), 32, replace=False), np.argsort(-np.abs(grad))[:32]]))
    L0 = bw["L"]
    worst = 0.0
    for j in pick:
        h = 1e-6 * w[j]
        vals = []
        for sgn in (1.0, -1.0):
            wj = w.copy()
            wj[j] += sgn * h
            with Graph.from_edges(src, dst, wj, n=g.n) as Gp:
                vals.append(Gp.adjoint_forward(part)["L"])
        fd = (vals[0] - vals[1]) / (2 * h)
        floor = 1e-14 * abs(L0) / h
        err = abs(fd - grad[j])
        assert err <= 1e-6 * abs(grad[j]) + floor, (j, fd, grad[j], floor)
        worst = max(worst, err / (1e-6 * abs(grad[j]) + floor))
    print(f"adjoint at 1M nodes: rel L1 vs CPU {_rel_l1(grad, rg):.2e}; FD worst {worst:.3f} of the bar "
          f"on {len(pick)} links")
