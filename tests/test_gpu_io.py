"""Output files and the drop-in command line."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu


def read_clu(path):
    lines = Path(path).read_bytes().split(b"\r\n")
    return np.array([int(x) - 1 for x in lines[1:] if x], dtype=np.int32)


def test_writer_byte_compatible(built_lib, tmp_path):
    """Given the reference's partition and code length, .tree/.clu are byte-identical."""
    from relaxmap_b200 import Graph
    part = read_clu(GOLDEN / "flow.ref.clu")
    with Graph.from_file(GOLDEN / "flow.net") as G:
        L = G.codelength(part)
        G.write_outputs(part, L, str(tmp_path), "/flow")
    assert (tmp_path / "flow.tree").read_bytes() == (GOLDEN / "flow.ref.tree").read_bytes()
    assert (tmp_path / "flow.clu").read_bytes() == (GOLDEN / "flow.ref.clu").read_bytes()


def test_cli_dropin(built_lib, tmp_path):
    exe = ROOT / "relaxmap_b200" / "ompRelaxmap"
    src = tmp_path / "in"
    src.mkdir()
    (src / "flow.net").write_bytes((GOLDEN / "flow.net").read_bytes())
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([str(exe), "1", str(src / "flow.net"), "1", "1", "1e-3", "0.0", "10", str(out), "prior"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "DONE: Code Length = 3.32773 in 4 modules, with 16 nodes." in r.stdout
    assert "Computed Code Length = 3.32773" in r.stdout
    tree = (out / "flow.tree").read_text().splitlines()
    assert tree[0] == "# Code length 3.32773 in 4 modules."
    assert len(tree) == 17
    clu = read_clu(out / "flow.clu")
    assert len(clu) == 16 and len(set(clu.tolist())) == 4


def test_cli_usage_and_bad_input(built_lib, tmp_path):
    exe = ROOT / "relaxmap_b200" / "ompRelaxmap"
    r = subprocess.run([str(exe), "1"], capture_output=True, text=True)
    assert r.returncode == 255 and "Call: ./ompRelaxmap" in r.stdout
    bad = tmp_path / "bad.net"
    bad.write_text("hello\n")
    r = subprocess.run([str(exe), "1", str(bad), "1", "1", "1e-3", "0.0", "10", str(tmp_path), "prior"],
                       capture_output=True, text=True)
    assert r.returncode == 255 and "not in Pajek format" in r.stdout


def test_invalid_arguments(built_lib):
    from relaxmap_b200 import Graph, RmxError
    with Graph.from_file(GOLDEN / "flow.net") as G:
        with pytest.raises(RmxError) as e:
            G.codelength(np.full(16, 99, dtype=np.int32))
        assert e.value.status == 1
    with pytest.raises(RmxError) as e:
        Graph.from_edges(np.array([0, 1]), np.array([1, 5]), n=3)
    assert e.value.status == 1


def test_cli_normal_mode_selflinks_and_attempts(built_lib, tmp_path):
    """The other argument forms of OmpRelaxmap.cpp:43-79: `normal` instead of
    `prior`, the optional `selflinks` (self links are still excluded, with the
    reference's message) and several attempts (the best is written)."""
    exe = ROOT / "relaxmap_b200" / "ompRelaxmap"
    net = tmp_path / "loops.txt"
    lines = (GOLDEN / "directNet_1k_sm_mu_03.txt").read_text().splitlines()
    lines += ["5 5", "7 7 2.0"]
    net.write_text("\n".join(lines) + "\n")
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([str(exe), "3", str(net), "4", "3", "1e-3", "0.0", "10", str(out), "normal", "selflinks"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "current version always excludes self links." in r.stdout
    assert "ignoring 2 self link(s)." in r.stdout
    done = [l for l in r.stdout.splitlines() if l.startswith("DONE: Code Length = ")]
    assert done, r.stdout
    L = float(done[-1].split("=")[1].split()[0])
    assert L <= 7.98793 * 1.005  # within the quality bar of the reference median on this graph
    assert (out / "loops.tree").exists() and (out / "loops.clu").exists()


def test_clu_round_trip(built_lib, tmp_path):
    """A partition written by rmx_write_outputs and read back with
    rmx_read_clu is the same partition with the same code length (resuming
    from a saved run)."""
    from relaxmap_b200 import Graph, read_clu as lib_read_clu
    with Graph.from_file(GOLDEN / "directNet_1k_sm_mu_03.txt") as G:
        r = G.optimize(seed=2)
        G.write_outputs(r["part"], r["L"], str(tmp_path), "/run")
        back = lib_read_clu(tmp_path / "run.clu", G.n)
        np.testing.assert_array_equal(back, r["part"])
        assert abs(G.codelength(back) - r["L"]) <= 1e-10 * r["L"]
