"""Device memory of closed graph handles stays in the library's block cache
(rmx_release_device_cache): after a handle closes its arenas stay allocated,
the next handle of the same size reuses them instead of allocating more, its
optimiser run is identical to the first handle's, and the release frees the
cached blocks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MB = 1 << 20


def test_handles_reuse_pooled_memory(built_lib):
    import torch
    from relaxmap_b200 import Graph, release_device_cache, synth
    g = synth.config_mid(seed=5, n=50_000)
    torch.cuda.init()
    release_device_cache()
    base = torch.cuda.mem_get_info()[0]
    results, held = [], []
    for _ in range(3):
        with Graph.from_edges(g.src, g.dst, g.w, n=g.n) as G:
            r = G.optimize(seed=7)
            results.append((r["part"].copy(), r["L"]))
        held.append(base - torch.cuda.mem_get_info()[0])  # measured after the handle closed
    for part, L in results[1:]:
        np.testing.assert_array_equal(part, results[0][0])
        assert L == results[0][1]
    # the two arenas of a 50K-node, ~1M-link handle are several hundred MB
    assert held[0] > 200 * MB, held
    assert max(held) - min(held) < 64 * MB, held
    release_device_cache()
    assert base - torch.cuda.mem_get_info()[0] < held[0] - 200 * MB
