"""The oracle pinned against the reference: golden vectors made by the reference
compiled from its own sources (tests/golden/make_golden.py), and, where the
reference harness was built (oracle/_ref), the reference run in-process."""
import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, golden


@pytest.mark.parametrize("name", FIXTURES)
def test_loader_matches_reference_map(oracle_mod, name):
    O = oracle_mod
    g = golden(name)
    path = GOLDEN / name
    ld = O.parse_pajek(path) if name.endswith(".net") else O.parse_txt(path)
    assert ld.n == int(g["n"])
    np.testing.assert_array_equal(ld.src, g["map_src"])
    np.testing.assert_array_equal(ld.dst, g["map_dst"])
    np.testing.assert_array_equal(ld.w, g["map_w"])
    np.testing.assert_array_equal(ld.node_w, g["node_w"])


@pytest.mark.parametrize("name", FIXTURES)
def test_initiate_bit_exact(oracle_mod, name):
    O = oracle_mod
    g = golden(name)
    prep = O.load(GOLDEN / name)
    np.testing.assert_array_equal(prep.off, g["off"])
    np.testing.assert_array_equal(prep.dst, g["dst"])
    st = O.initiate(prep)
    np.testing.assert_array_equal(st["p"], g["p"])
    np.testing.assert_array_equal(st["f"], g["f"])
    np.testing.assert_array_equal(st["exit"], g["exit"])
    np.testing.assert_array_equal(st["dangling"], g["dangling"])
    assert st["L0"] == float(g["L0"])
    assert st["all_log_all"] == float(g["all_log_all"])


@pytest.mark.parametrize("name", FIXTURES)
def test_codelength_of_reference_partition(oracle_mod, name):
    O = oracle_mod
    g = golden(name)
    prep = O.load(GOLDEN / name)
    st = O.initiate(prep)
    L = O.codelength(prep, st, g["part_seed1"])
    assert abs(L - float(g["part_seed1_codelength"])) <= 1e-12 * max(1.0, abs(L))
    # the reference's own final "Computed Code Length" for that run
    assert abs(L / np.log(2) - g["final_L_computed_bits"][0][0]) < 1e-9


@pytest.mark.parametrize("name", FIXTURES)
def test_convert_bit_exact(oracle_mod, name):
    O = oracle_mod
    g = golden(name)
    prep = O.load(GOLDEN / name)
    st = O.initiate(prep)
    cv = O.convert(prep.n, prep.off, prep.dst, st["f"], g["part_seed1"])
    assert cv["n_sn"] == len(g["sn_modidx"])
    np.testing.assert_array_equal(np.nonzero(cv["sn_of_mod"] >= 0)[0], g["sn_modidx"])
    for k in ("out_off", "out_dst", "out_f", "in_off", "in_src", "in_f"):
        np.testing.assert_array_equal(cv[k], g["sn_" + k], err_msg=k)


def test_known_answers():
    """Known answers of the bundled data (reference runs, bits)."""
    g = golden("flow.net")
    assert np.all(np.round(g["final_L_bits"], 5) == 3.32773)
    assert np.all(g["final_n_modules"] == 4)
    g = golden("directNet_1k_sm_mu_03.txt")
    assert round(float(np.median(g["final_L_bits"])), 5) == 7.98793


def test_mt19937_stream(oracle_mod):
    """The bundled MTRand seeding: with seed s the reference's order matches."""
    import ctypes as C

    class MT(C.Structure):
        _fields_ = [("state", C.c_uint32 * 624), ("left", C.c_int), ("next", C.c_int)]

    L = oracle_mod.lib()
    m = MT()
    L.rmxo_mt_seed(C.byref(m), C.c_uint32(7))
    # first draws of MTRand(7).randInt() and randInt(15), from the reference header
    assert [L.rmxo_mt_rand(C.byref(m)) for _ in range(4)] == [22671274, 109824311, 1824471040, 3737574225]
    L.rmxo_mt_seed(C.byref(m), C.c_uint32(7))
    assert [L.rmxo_mt_randint(C.byref(m), 15) for _ in range(6)] == [10, 7, 0, 1, 12, 10]


@pytest.mark.parametrize("name", ["flow.net", "directNet_1k_sm_mu_03.txt", "small_planted.txt"])
@pytest.mark.parametrize("prior", [0, 1])
def test_sequential_sweeps_replay_reference(oracle_mod, name, prior):
    """The oracle's one-thread sweeps (move / prioritize_move with the bundled
    MT19937) replay the reference's trajectory exactly."""
    O = oracle_mod
    if O.reflib() is None:
        pytest.skip("reference harness not built")
    prep = O.load(GOLDEN / name)
    st = O.initiate(prep)
    for seed in (1, 7):
        Lr, pr, nr = ref_sweeps(O, name, seed, prior)
        Lo, po, no = O.node_sweeps(prep, st, seed, prior, 0.0, 1e-3, 10)
        assert Lr == Lo and nr == no
        np.testing.assert_array_equal(pr, po)


def ref_sweeps(O, name, seed, prior):
    """A fresh reference network per run (the sweeps change its state)."""
    R = O.Ref(path=GOLDEN / name)
    R.prepare(1)
    return R.node_sweeps(seed, prior, 0.0, 1e-3, 10)


def test_evaluate_matches_sweep_decision(oracle_mod):
    """rmxo_evaluate gives the same first decision the sequential sweep takes:
    from singletons, the first node of the random order moves to the module
    evaluate() picks for it."""
    O = oracle_mod
    prep = O.load(GOLDEN / "flow.net")
    st = O.initiate(prep)
    n = prep.n
    units = dict(out_off=prep.off, out_dst=prep.dst, out_f=st["f"], in_off=st["in_off"], in_src=st["in_src"],
                 in_f=st["in_f"], p=st["p"], tw=prep.tw, dsize=st["dsize"], exit=st["exit"])
    mod = np.arange(n, dtype=np.int32)
    ms = O.module_stats(n, st["p"], prep.tw, st["dsize"], prep.off, prep.dst, st["f"], mod)
    bm, bd = O.evaluate(units, mod, ms, float(ms["exit"].sum()))
    assert np.all(bd <= 0)
    # singletons everywhere: every node has a strictly improving merge
    assert np.all(bm >= 0)
