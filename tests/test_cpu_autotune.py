"""Launch tuning without a GPU: rmx_get_tuning / rmx_set_tuning through the
C ABI (process-wide values, no device call), and the autotuner's search,
result check and per-device cache driven by fake measurements."""
import json

import pytest


@pytest.fixture
def restore_tuning(built_lib):
    from relaxmap_b200 import get_tuning, set_tuning
    before = get_tuning()
    yield
    set_tuning(**before)


def test_tuning_abi_defaults_and_validation(restore_tuning):
    from relaxmap_b200 import RmxError, get_tuning, set_tuning
    from relaxmap_b200.autotune import DEFAULTS, KNOBS
    assert get_tuning() == DEFAULTS
    for k, cands in KNOBS.items():
        assert DEFAULTS[k] in cands
    assert set_tuning(eval_mid_grid=12, eval_reg_grid=16) == dict(DEFAULTS, eval_mid_grid=12, eval_reg_grid=16)
    assert get_tuning() == dict(DEFAULTS, eval_mid_grid=12, eval_reg_grid=16)
    for bad in (0, 65, -3):
        with pytest.raises(RmxError) as e:
            set_tuning(eval_warp_grid=bad)
        assert e.value.status == 1  # RMX_ERR_INVALID
    assert get_tuning() == dict(DEFAULTS, eval_mid_grid=12, eval_reg_grid=16)  # unchanged by a rejected call
    with pytest.raises(ValueError):
        set_tuning(eval_hub_grid=2)
    # degree bounds: ordered, each within its bin's table limit
    assert set_tuning(warp_max_degree=64, mid_max_degree=64)["mid_max_degree"] == 64
    for bad in ({"warp_max_degree": 31}, {"warp_max_degree": 129}, {"mid_max_degree": 63},
                {"mid_max_degree": 513}, {"block_max_degree": 1025}, {"large_max_degree": 1000},
                {"large_max_degree": 4097}, {"hub_partition_links": 63}, {"hub_partition_links": (1 << 30) + 1}):
        with pytest.raises(RmxError) as e:
            set_tuning(**bad)
        assert e.value.status == 1
    assert get_tuning() == dict(DEFAULTS, eval_mid_grid=12, eval_reg_grid=16, warp_max_degree=64,
                                mid_max_degree=64)


def _quadratic(opt, L=1.0, calls=None):
    def measure(cfg):
        if calls is not None:
            calls.append(dict(cfg))
        return 100.0 + 10.0 * sum((cfg[k] - opt[k]) ** 2 for k in opt), L  # steps well above the margin
    return measure


def test_tune_finds_the_fastest_setting():
    from relaxmap_b200.autotune import DEFAULTS, tune
    opt = {"eval_mid_grid": 12, "eval_block_grid": 6, "eval_large_grid": 2, "eval_warp_grid": 3, "eval_reg_grid": 4}
    calls = []
    r = tune(_quadratic(opt, calls=calls))
    assert r["tuning"] == dict(DEFAULTS, **opt)  # the bin bounds do not change the modelled time
    assert r["ms"] == 100.0
    assert r["baseline_ms"] == 100.0 + 10.0 * sum((DEFAULTS[k] - opt[k]) ** 2 for k in opt)
    assert r["timed_settings"] == len(calls)
    assert calls[0] == DEFAULTS  # the baseline is timed first


def test_tune_times_each_setting_once():
    """After a knob moves, coordinate descent meets earlier settings again
    (the old value of that knob, or a second pass): they are not re-timed."""
    from relaxmap_b200.autotune import DEFAULTS, tune
    opt = {"eval_mid_grid": 4, "eval_warp_grid": 2}  # the other knobs keep their defaults
    knobs = {"eval_mid_grid": (4, 8), "eval_warp_grid": (2, 3)}
    for passes, distinct in ((1, 3), (3, 4)):  # the second pass adds (mid 8, warp 2) only
        calls = []
        r = tune(_quadratic(opt, calls=calls), knobs=knobs, passes=passes)
        assert r["tuning"] == dict(DEFAULTS, **opt)
        keys = [tuple(sorted(c.items())) for c in calls]
        assert len(keys) == len(set(keys)) == r["timed_settings"] == distinct


def test_tune_keeps_settings_within_the_noise_margin():
    from relaxmap_b200.autotune import DEFAULTS, tune

    def measure(cfg):  # every other setting is 0.5% faster: below the 1% margin
        return (100.0 if cfg == DEFAULTS else 99.5), 3.0
    r = tune(measure)
    assert r["tuning"] == DEFAULTS and r["ms"] == 100.0


def test_tune_rejects_a_setting_that_changes_the_result():
    from relaxmap_b200.autotune import TuningError, tune

    def measure(cfg):
        return 10.0, (2.0 if cfg["eval_block_grid"] == 6 else 1.0)
    with pytest.raises(TuningError, match="eval_block_grid=6"):
        tune(measure)


def test_tune_rejects_unknown_knobs():
    from relaxmap_b200.autotune import tune
    with pytest.raises(ValueError):
        tune(_quadratic({}), knobs={"eval_hub_grid": (1, 2)})


def test_save_and_load_per_device(tmp_path, restore_tuning):
    from relaxmap_b200 import get_tuning
    from relaxmap_b200.autotune import DEFAULTS, load, save
    tuned = dict(DEFAULTS, eval_mid_grid=16, eval_warp_grid=4)
    p = tmp_path / "tuning.json"
    save({"device": "B200|148 SMs", "tuning": tuned, "ms": 90.0, "baseline_ms": 100.0,
          "graph": {"nodes": 10, "links": 20}}, p)
    assert json.loads(p.read_text())["format"] == 1
    assert load(p, device="H100|132 SMs") is None  # another device: nothing applied
    assert get_tuning() == DEFAULTS
    assert load(p, device="B200|148 SMs") == tuned
    assert get_tuning() == tuned
    p.write_text(json.dumps({"format": 7, "device": "B200|148 SMs", "tuning": tuned}))
    with pytest.raises(ValueError):
        load(p, device="B200|148 SMs")


def test_cli_tuning_flag(tmp_path, restore_tuning):
    """ompRelaxmap ... [selflinks] --tuning=<file> applies a tuning file before
    the network is read (the missing network here stops the run there, so no
    device is needed); a file with an invalid value is rejected (exit -1)
    without changing the setting."""
    from relaxmap_b200 import cli, get_tuning
    from relaxmap_b200.autotune import DEFAULTS
    good = tmp_path / "tuning.json"
    good.write_text(json.dumps({"format": 1, "device": "any", "tuning": dict(DEFAULTS, eval_mid_grid=12,
                                                                              eval_reg_grid=6)}))
    args = ["ompRelaxmap", "1", str(tmp_path / "missing.txt"), "1", "1", "1e-3", "0.0", "10", str(tmp_path),
            "prior", "selflinks"]
    assert cli(args + [f"--tuning={good}"]) == -1  # the network file is missing
    assert get_tuning() == dict(DEFAULTS, eval_mid_grid=12, eval_reg_grid=6)
    bad = tmp_path / "bad.json"
    bad.write_text('{"tuning": {"eval_warp_grid": 0}}')
    assert cli(args + [f"--tuning={bad}"]) == -1
    assert get_tuning() == dict(DEFAULTS, eval_mid_grid=12, eval_reg_grid=6)
    assert cli(args + [f"--tuning={tmp_path / 'none.json'}"]) == -1
