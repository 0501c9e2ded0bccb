"""Launch tuning on the device changes time, not results: optimiser runs under
extreme grid caps of the move-evaluation bins (one block per SM, and many)
and under other degree bounds of the bins (every unit above 32 links in the
hub bin's global tables; narrow warp and mid bins; empty bins) give the same
partition and code length bit for bit as the defaults, both on direct
launches and on sweep CUDA graphs captured after the change; the autotuner
runs end to end, restores the setting it found, and its saved result applies
on this device."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def graph(built_lib):
    from relaxmap_b200 import Graph, get_tuning, set_tuning, synth
    g = synth.config_mid(seed=9, n=20_000)  # units in the register, warp, mid and block bins
    before = get_tuning()
    with Graph.from_edges(g.src, g.dst, g.w, n=g.n) as G:
        yield G
    set_tuning(**before)


def test_launch_shape_does_not_change_results(graph):
    from relaxmap_b200 import TUNING_FIELDS, set_tuning
    from relaxmap_b200.autotune import DEFAULTS
    G = graph
    ref = G.optimize(seed=3)
    caps = [f for f in TUNING_FIELDS if f.endswith("_grid")]
    for cfg in ({f: 1 for f in caps},
                {"eval_mid_grid": 16, "eval_block_grid": 8, "eval_large_grid": 3, "eval_warp_grid": 8,
                 "eval_reg_grid": 16},
                DEFAULTS,
                dict(DEFAULTS, warp_max_degree=32, mid_max_degree=32, block_max_degree=32, large_max_degree=32),
                dict(DEFAULTS, warp_max_degree=48, mid_max_degree=200, block_max_degree=200, large_max_degree=700),
                dict(DEFAULTS, warp_max_degree=128, mid_max_degree=128, block_max_degree=1024,
                     large_max_degree=1024),
                dict(DEFAULTS, mid_max_degree=256, block_max_degree=256, large_max_degree=256, hub_partition_links=64),
                DEFAULTS):
        set_tuning(**cfg)
        for _ in range(2):  # the second run replays the sweep graphs captured by the first
            G.reset_flow()
            r = G.optimize(seed=3)
            np.testing.assert_array_equal(r["part"], ref["part"])
            assert r["L"] == ref["L"]


def test_autotune_end_to_end(graph, tmp_path):
    from relaxmap_b200 import get_tuning
    from relaxmap_b200.autotune import DEFAULTS, device_key, load, save, tune_graph
    set_tuning_before = get_tuning()
    res = tune_graph(graph, seed=2, reps=1, passes=1,
                     knobs={"eval_mid_grid": (4, 8), "eval_warp_grid": (2, 3)})
    assert get_tuning() == set_tuning_before  # tuning leaves the process setting alone
    assert res["timed_settings"] == 3 and res["ms"] > 0 and res["baseline_ms"] > 0
    assert set(res["tuning"]) == set(DEFAULTS)
    assert res["device"] == device_key()
    p = tmp_path / "tuning.json"
    save(res, p)
    assert load(p) == res["tuning"]
    assert get_tuning() == res["tuning"]
