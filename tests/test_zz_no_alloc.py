"""rmx_steady_state_noalloc: the stationary flow for callers that cannot
allocate device memory (a framework whose pool owns the whole device under a
fixed budget, or a path that must not synchronise the device on an
allocation). The caller provides every input and output on the device; the
library uses only its own fixed in-library scratch.

Checked through the C ABI on two calls in a row against the existing entry
point (rmx_initiate) and against the reference's own flow (the golden vectors
made by running the reference), both within the flow tolerance used elsewhere
(1e-12 relative L1); and on a graph with in-degree hubs, where the two entry
points sum those rows in different orders (iteration count within one).
Collected last so that a failure here leaves every other test run."""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def rel_l1(a, b):
    return np.abs(a - b).sum() / np.abs(b).sum()


def device_inputs(G, torch):
    """Row-normalised CSC, teleport weights and dangling flags of graph G,
    built on the host and copied to device buffers owned by the test."""
    off, dst, w, tw = G.links()
    n, m = G.n, len(dst)
    src = np.repeat(np.arange(n), np.diff(off))
    rowsum = np.zeros(n)
    np.add.at(rowsum, src, w)
    wn = w / rowsum[src]
    order = np.argsort(dst, kind="stable")
    in_off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(dst, minlength=n), out=in_off[1:])
    dang = (np.diff(off) == 0).astype(np.uint8)
    dev = dict(in_off=torch.from_numpy(in_off).cuda(), in_src=torch.from_numpy(src[order].astype(np.int32)).cuda(),
               in_w=torch.from_numpy(wn[order].copy()).cuda(), tw=torch.from_numpy(tw).cuda(),
               dang=torch.from_numpy(dang).cuda())
    return n, m, dev


def run_noalloc(torch, n, m, dev, ref, exact_iters):
    from relaxmap_b200._lib import steady_state_noalloc
    stream = torch.cuda.current_stream()
    for call in range(2):  # the shared scratch keeps the previous call's contents
        p = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        iters = torch.zeros(1, dtype=torch.int32, device="cuda")
        steady_state_noalloc(n, m, dev["in_off"].data_ptr(), dev["in_src"].data_ptr(), dev["in_w"].data_ptr(),
                             dev["tw"].data_ptr(), dev["dang"].data_ptr(), p.data_ptr(), iters.data_ptr(),
                             stream.cuda_stream)
        stream.synchronize()
        got = p.cpu().numpy()
        assert np.all(np.isfinite(got)), call
        assert rel_l1(got, ref["p"]) <= 1e-12, (call, rel_l1(got, ref["p"]))
        if exact_iters:
            assert int(iters.item()) == ref["iters"]
        else:
            assert abs(int(iters.item()) - ref["iters"]) <= 1
    return got


@pytest.mark.parametrize("name", ["small_planted.txt", "flow.net", "directNet_1k_sm_mu_03.txt"])
def test_noalloc_matches_initiate(built_lib, name):
    import torch

    from relaxmap_b200 import Graph, RmxError
    from relaxmap_b200._lib import steady_state_noalloc

    with Graph.from_file(GOLDEN / name) as G:
        ref = G.initiate()
        n, m, dev = device_inputs(G, torch)
    got = run_noalloc(torch, n, m, dev, ref, exact_iters=True)
    with np.load(GOLDEN / (name + ".ref.npz")) as z:  # the reference's own flow
        assert rel_l1(got, z["p"]) <= 1e-12
    with pytest.raises(RmxError) as e:
        steady_state_noalloc(1 << 21, m, dev["in_off"].data_ptr(), dev["in_src"].data_ptr(), dev["in_w"].data_ptr(),
                             dev["tw"].data_ptr(), dev["dang"].data_ptr(), 1, 0, 0)
    assert e.value.status == 1


def test_noalloc_in_degree_hubs(built_lib):
    """A graph whose in-degree hubs rmx_initiate sums in chunks."""
    import torch

    from relaxmap_b200 import Graph
    rng = np.random.default_rng(8)
    n = 20000
    src = [rng.integers(0, n, 8 * n)]
    dst = [rng.integers(0, n, 8 * n)]
    for hub in range(4):
        src.append(rng.integers(0, n, 6000))
        dst.append(np.full(6000, hub))
    src, dst = np.concatenate(src), np.concatenate(dst)
    with Graph.from_edges(src, dst, rng.uniform(1, 2, len(src)), n=n) as G:
        ref = G.initiate()
        n, m, dev = device_inputs(G, torch)
    run_noalloc(torch, n, m, dev, ref, exact_iters=False)
