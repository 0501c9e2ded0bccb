"""Pins the CPU adjoint (oracle/adjoint.py) against the reference itself.

The reference has no gradient, so the pin is its own forward model: the code
length it computes (Network::initiate, then calculateCodeLength on a fixed
partition) after perturbing one link weight by +-h, h = 1e-6 relative, for 64
links; and, for the teleportation probability it fixes at 0.15, centred
differences of the CPU forward model, whose value at 0.15 equals the
reference's code length to 1e-12."""
import numpy as np
import pytest

from conftest import GOLDEN

O = pytest.importorskip("oracle.oracle")
AD = pytest.importorskip("oracle.adjoint")


def _ref_partition(ld):
    R = O.Ref(loaded=ld)
    R.prepare(1)
    return np.asarray(R.partition(seed=1, threads=1)["part"], dtype=np.int32)


def _ref_L(ld, part, w):
    R = O.Ref(loaded=O.Loaded(ld.n, ld.names, ld.node_w, ld.tot_w, ld.src, ld.dst, w))
    R.prepare(1)
    R.set_partition(part)
    return R.calc_codelength()


@pytest.mark.parametrize("name,n_links", [("directNet_1k_sm_mu_03.txt", 64), ("flow.net", 8)])
def test_adjoint_matches_reference_differences(built_lib, name, n_links):
    if O.reflib() is None:
        pytest.skip("reference harness not built")
    path = GOLDEN / name
    ld = O.parse_pajek(path) if name.endswith(".net") else O.parse_txt(path)
    pr = O.prepare(ld)
    part = _ref_partition(ld)
    bw = AD.backward(pr.off, pr.dst, pr.w, pr.tw, part)
    assert abs(bw["L"] - _ref_L(ld, part, ld.w)) <= 1e-12 * abs(bw["L"])
    keep = np.nonzero((ld.w > 0) & (ld.src != ld.dst))[0]  # prepared link j is map entry keep[j]
    rng = np.random.default_rng(7)
    for j in rng.choice(len(pr.dst), min(n_links, len(pr.dst)), replace=False):
        k = keep[j]
        h = 1e-6 * ld.w[k]
        wp, wm = ld.w.copy(), ld.w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (_ref_L(ld, part, wp) - _ref_L(ld, part, wm)) / (2 * h)
        # centred differences carry ~1e-14 / h of rounding: absolute 2e-8, relative 1e-3
        assert abs(fd - bw["dL_dw"][j]) <= 2e-8 + 1e-3 * abs(bw["dL_dw"][j]), (j, fd, bw["dL_dw"][j])


def test_adjoint_teleportation_derivative(built_lib):
    pr = O.load(GOLDEN / "directNet_1k_sm_mu_03.txt")
    part = np.arange(pr.n, dtype=np.int32) // 25  # 40 blocks of consecutive ids
    bw = AD.backward(pr.off, pr.dst, pr.w, pr.tw, part, t=0.2)
    h = 1e-6
    fd = (AD.forward(pr.off, pr.dst, pr.w, pr.tw, part, 0.2 + h)["L"] -
          AD.forward(pr.off, pr.dst, pr.w, pr.tw, part, 0.2 - h)["L"]) / (2 * h)
    assert abs(fd - bw["dL_dt"]) <= 1e-6 * abs(bw["dL_dt"])
