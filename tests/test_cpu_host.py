"""Host-side logic without a GPU: the C ABI library loads and exports every
declared symbol, the loaders follow the reference's parsing rules, and input
errors map to status codes."""
import re

import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, ROOT, golden


def test_exports_match_header(built_lib):
    import ctypes
    from relaxmap_b200 import EXPORTS
    hdr = (ROOT / "include" / "relaxmap_b200.h").read_text()
    declared = set(re.findall(r"\b(rmx_\w+)\s*\(", hdr))
    assert declared == set(EXPORTS)
    L = ctypes.CDLL(str(built_lib))
    for name in declared:
        assert hasattr(L, name), name


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("threads", [1, 4])
def test_parse_matches_reference_loader(built_lib, name, threads):
    from relaxmap_b200 import parse_file
    g = golden(name)
    d = parse_file(GOLDEN / name, threads=threads)
    assert d["n"] == int(g["n"])
    acc = {}
    for a, b, x in zip(d["src"].tolist(), d["dst"].tolist(), d["w"].tolist()):
        acc[(a, b)] = acc.get((a, b), 0.0) + x
    ref = {(a, b): x for a, b, x in zip(g["map_src"].tolist(), g["map_dst"].tolist(), g["map_w"].tolist()) if a != b}
    assert acc == ref
    np.testing.assert_array_equal(d["node_w"], g["node_w"])


def _cmp_oracle(path, oracle_mod, threads=(1, 3)):
    from relaxmap_b200 import parse_file
    O = oracle_mod
    ld = O.parse_pajek(path) if str(path).endswith(".net") else O.parse_txt(path)
    for t in threads:
        d = parse_file(path, threads=t)
        assert d["n"] == ld.n
        acc = {}
        for a, b, x in zip(d["src"].tolist(), d["dst"].tolist(), d["w"].tolist()):
            acc[(a, b)] = acc.get((a, b), 0.0) + x
        ref = {(a, b): x for a, b, x in zip(ld.src.tolist(), ld.dst.tolist(), ld.w.tolist()) if a != b}
        assert acc == ref
        n_self = sum(1 for a, b, x in zip(ld.src.tolist(), ld.dst.tolist(), ld.w.tolist()) if a == b and x > 0)
        assert d["n_self"] == n_self
    return ld


def test_edge_list_quirks(built_lib, oracle_mod, tmp_path):
    """Comments, CRLF, weights, duplicates, self-links, sparse / negative ids,
    and a blank line re-reading the previous token (a phantom self-link)."""
    p = tmp_path / "q.txt"
    p.write_bytes(b"# comment\n5 9 2.5\r\n9 5\n\n5 9 0.5\n-3 5 1e-1\n7 7 4\n  100\t5 3\n\n")
    ld = _cmp_oracle(p, oracle_mod)
    # a blank line after "9 5" re-reads "" (node 0); after "100 5 3" it re-reads "3"
    assert ld.names == ["-3", "0", "3", "5", "7", "9", "100"]


def test_weights_parse_like_strtod(built_lib, oracle_mod, tmp_path):
    """Weights read with the decimal fast path (plain decimals with a mantissa
    below 2^53 and at most 22 fractional digits) and with strtod (all other
    forms) equal the correctly rounded values of the oracle, weight by weight
    (every line its own link)."""
    rng = np.random.default_rng(8)
    lines = []
    for i in range(30000):
        k = rng.integers(0, 10)
        digits = "".join(rng.choice(list("0123456789"), size=rng.integers(1, 21)))
        cut = int(rng.integers(0, len(digits) + 1))
        sign = ["", "-", "+"][rng.integers(0, 3)]
        if k < 6:    # plain decimals: both sides of the 2^53 and 22-fraction-digit limits
            w = sign + digits[:cut] + "." + digits[cut:] if k < 4 else sign + digits
        elif k == 6:  # long fractions, leading zeros
            w = sign + "0." + "0" * int(rng.integers(0, 25)) + digits
        elif k == 7:  # exponents
            w = sign + digits[:cut] + "." + digits[cut:] + "e" + str(int(rng.integers(-30, 30)))
        elif k == 8:  # trailing characters, bare point, infinities, hexadecimal (C99 strtod reads 0x1p3 as 8)
            w = [sign + digits + "x", ".", sign + ".5", "inf", "-infinity", "0x1p3", sign + digits + ".e",
                 "-0x.8p1"][rng.integers(0, 8)]
        else:
            w = sign + digits[:cut] + "." + digits[cut:] + "abc"
        lines.append(f"{2 * i} {2 * i + 1} {w}")
    p = tmp_path / "weights.txt"
    p.write_text("\n".join(lines) + "\n")
    _cmp_oracle(p, oracle_mod, threads=(1,))


def test_edge_list_large_threads(built_lib, oracle_mod, tmp_path):
    rng = np.random.default_rng(2)
    lines = []
    for i in range(120000):
        r = rng.random()
        if r < 0.01:
            lines.append("")
        elif r < 0.02:
            lines.append("# c")
        elif r < 0.5:
            lines.append(f"{rng.integers(0, 5000)} {rng.integers(0, 5000)}")
        else:
            lines.append(f"{rng.integers(0, 5000)}\t{rng.integers(0, 5000)}\t{rng.uniform(-1, 5)!r}")
    p = tmp_path / "big.txt"
    p.write_text("\n".join(lines) + "\n")
    _cmp_oracle(p, oracle_mod)


def test_edge_list_quirks_at_range_boundaries(built_lib, oracle_mod, tmp_path):
    """Byte ranges of the parallel parse start at line starts; with four lines
    in ten a blank, whitespace-only, bare-CR, one-token or comment line, many
    ranges open on a blank-like line that re-reads the stream state carried in
    (the last non-comment line's third token): 1, 5 and 13 of the range starts
    at 7, 16 and 64 threads follow a line with a weight, so a lost state
    changes the edge map."""
    rng = np.random.default_rng(11)
    kinds = rng.choice(8, size=110000, p=[0.15, 0.05, 0.05, 0.05, 0.10, 0.25, 0.30, 0.05])
    ids = rng.integers(0, 3000, size=(110000, 2))
    wts = rng.uniform(0.0, 4.0, size=110000)
    lines = []
    for k, (a, b), x in zip(kinds.tolist(), ids.tolist(), wts.tolist()):
        lines.append(["", " \t ", "\r", f"{a}", f"# {a} {b} 7", f"{a} {b}",
                      f"{a}\t{b}\t{x!r}", f"{a} {b} {x:.3f}\r"][k])
    p = tmp_path / "dense_quirks.txt"
    p.write_text("\n".join(lines) + "\n")
    assert p.stat().st_size > (1 << 20)  # large enough for the multi-range parse
    _cmp_oracle(p, oracle_mod, threads=(1, 2, 7, 16, 64))


def test_edge_list_ids_across_the_64_bit_range(built_lib, oracle_mod, tmp_path):
    """Ids at both ends of the 64-bit range: sparse, so renumbered by sorting,
    and their span does not fit a signed difference."""
    p = tmp_path / "wide.txt"
    p.write_text("-9223372036854775808 9223372036854775807 2\n9223372036854775807 0\n"
                 "0 -9223372036854775808 0.5\n5 5 1\n-1 0\n")
    ld = _cmp_oracle(p, oracle_mod)
    assert ld.names == ["-9223372036854775808", "-1", "0", "5", "9223372036854775807"]


def test_pajek_quirks(built_lib, oracle_mod, tmp_path):
    p = tmp_path / "q.net"
    p.write_text('*Vertices 5\n1 "a b" 2.0\n2 "c"\n3 d 0.5\n4\n5 "e" -1\n*Arcs\n1 2\n2 3 0.5\n1 2 1.5\n3 3 2\n\n5 1\n')
    ld = _cmp_oracle(p, oracle_mod)
    assert ld.names == ["a b", "c", "d", "4", "e"]
    np.testing.assert_array_equal(ld.node_w, [2.0, 1.0, 0.5, 1.0, 1.0])


def _pajek_text(rng, n, n_arcs):
    vert = [f"*Vertices {n}"] + [f'{i + 1} "v{i + 1}"' for i in range(n)]
    kinds = rng.choice(6, size=n_arcs, p=[0.15, 0.05, 0.05, 0.25, 0.40, 0.10])
    ids = rng.integers(1, n + 1, size=(n_arcs, 2))
    wts = rng.uniform(0.0, 4.0, size=n_arcs)
    arcs = [["", " \t ", "\r", f"{a} {b}", f"{a}\t{b}\t{x!r}", f"{a} {b} {x:.3f}\r"][k]
            for k, (a, b), x in zip(kinds.tolist(), ids.tolist(), wts.tolist())]
    # a blank line right after the header re-reads the header token
    return vert + ["*Arcs", ""] + arcs


def test_pajek_arcs_at_range_boundaries(built_lib, oracle_mod, tmp_path):
    """The arcs section is parsed in byte ranges on all threads; each range
    starts with the stream state of the line before it (its third token or
    ""; the header token for the first), which blank, whitespace-only and
    bare-CR lines re-read as a self-link."""
    rng = np.random.default_rng(5)
    lines = _pajek_text(rng, 3000, 150000)
    p = tmp_path / "arcs.net"
    p.write_text("\n".join(lines) + "\n")
    assert len("\n".join(lines[3002:])) > (1 << 20)  # the arcs section alone takes the multi-range parse
    _cmp_oracle(p, oracle_mod, threads=(1, 2, 7, 16, 64))


def test_pajek_first_bad_link_in_file_order(built_lib, tmp_path):
    from relaxmap_b200 import RmxError, parse_file
    rng = np.random.default_rng(6)
    lines = _pajek_text(rng, 3000, 150000)
    lines[3002 + 60000] = "1 3001"
    lines[3002 + 140000] = "3002 5 1.5"
    p = tmp_path / "bad_arcs.net"
    p.write_text("\n".join(lines) + "\n")
    for t in (1, 8, 64):
        with pytest.raises(RmxError) as e:
            parse_file(p, threads=t)
        assert e.value.status == 3 and "link 1 3001 outside 1..3000" in str(e.value)


def test_errors_without_device(built_lib, tmp_path):
    from relaxmap_b200 import Graph, RmxError, parse_file
    with pytest.raises(RmxError) as e:
        parse_file(tmp_path / "missing.txt")
    assert e.value.status == 2  # RMX_ERR_IO
    bad = tmp_path / "bad.net"
    bad.write_text("*Network x\n")
    with pytest.raises(RmxError) as e:
        Graph.from_file(bad)
    assert e.value.status == 3  # RMX_ERR_FORMAT (the reference exits -1)
    bad.write_text("*Vertices 2\n1\n2\n*Edges\n1 3\n")
    with pytest.raises(RmxError) as e:
        parse_file(bad)
    assert e.value.status == 3
    bad.write_text("*Vertices 3\n1\n2\n3\n*ARCS\n")
    with pytest.raises(RmxError) as e:
        parse_file(bad)
    assert e.value.status == 3


def test_synth_deterministic():
    from relaxmap_b200 import synth
    a = synth.config_small(seed=42)
    b = synth.config_small(seed=42)
    np.testing.assert_array_equal(a.src, b.src)
    np.testing.assert_array_equal(a.dst, b.dst)
    assert a.n == 1000 and 15 < a.m / a.n < 21
    r = synth.rmat(10, 16, seed=1)
    assert r.n == 1024 and np.all(r.src != r.dst)
    assert len(np.unique(r.src.astype(np.int64) * r.n + r.dst)) == r.m


def test_batch_host_validation(built_lib):
    """rmx_batch_create only copies and checks the graphs in host memory: ids
    local to each graph, at least one node per graph; wave budgets positive.
    Nothing here touches a device."""
    from relaxmap_b200 import Batch, RmxError
    ok = [(3, np.array([0, 1], np.int32), np.array([1, 2], np.int32), None),
          (2, np.array([1], np.int32), np.array([0], np.int32), np.array([2.5]))]
    with Batch(ok) as B:
        info = B.info()
        assert info == {"graphs": 2, "waves": 0, "instances": 0, "device_ms": 0.0}
        with pytest.raises(RmxError) as e:
            B.set_wave(0, 10)
        assert e.value.status == 1
        B.set_wave(1 << 20, 1 << 20)
        assert list(B.offsets) == [0, 3, 5]
    for bad in ([(3, np.array([0, 3], np.int32), np.array([1, 2], np.int32), None)],  # id beyond its graph
                [(0, np.zeros(0, np.int32), np.zeros(0, np.int32), None)],           # empty graph
                [(2, np.array([-1], np.int32), np.array([0], np.int32), None)]):     # negative id
        with pytest.raises(RmxError) as e:
            Batch(bad)
        assert e.value.status == 1


def test_lpt_weights_edge_cases():
    from relaxmap_b200.sharding import lpt_assign
    parts = lpt_assign([5.0], 4)  # more ranks than graphs: some ranks get none
    assert [len(p) for p in parts] == [1, 0, 0, 0]
    parts = lpt_assign([1.0, 1.0, 1.0, 1.0], 2)
    assert sorted(len(p) for p in parts) == [2, 2]


def test_header_is_c99_and_links_from_c(built_lib, tmp_path):
    """include/relaxmap_b200.h compiles as strict C99 and a C program links
    against the library and calls its device-free entry points (what a C
    caller of the ABI does); skipped without gcc."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no gcc")
    prog = tmp_path / "abi.c"
    prog.write_text('#include <stdio.h>\n#include "relaxmap_b200.h"\n'
                    "int main(void) {\n"
                    "    rmx_tuning t;\n"
                    "    rmx_opts o;\n"
                    "    rmx_opts_default(&o);\n"
                    "    if (rmx_get_tuning(&t) != RMX_OK) return 1;\n"
                    "    t.eval_warp_grid = 0;\n"
                    "    if (rmx_set_tuning(&t) != RMX_ERR_INVALID) return 2;\n"
                    "    printf(\"%s|%d|%u\\n\", rmx_version(), t.eval_mid_grid, o.seed);\n"
                    "    return 0;\n}\n")
    exe = tmp_path / "abi"
    lib_dir = built_lib.parent
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", str(ROOT / "include"), str(prog),
                    "-L", str(lib_dir), "-lrelaxmap_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert out.startswith("relaxmap_b200")


def test_parse_size_query_then_fill(built_lib, tmp_path):
    """rmx_parse_file's size query keeps its parse for the fill call that
    follows (one parse for the pair); a file changed in between is parsed
    again, so the fill returns the new contents."""
    import ctypes as C
    import os
    from relaxmap_b200 import lib
    L = lib()
    p = tmp_path / "g.txt"
    p.write_text("1 2 1.5\n2 3 2.5\n")
    n, m, ns = C.c_int32(), C.c_int64(), C.c_int64()

    def query():
        assert L.rmx_parse_file(str(p).encode(), 1, C.byref(n), C.byref(m), C.byref(ns), None, None, None, None) == 0

    def fill():
        src, dst = (C.c_int32 * m.value)(), (C.c_int32 * m.value)()
        w, nw = (C.c_double * m.value)(), (C.c_double * n.value)()
        assert L.rmx_parse_file(str(p).encode(), 1, C.byref(n), C.byref(m), C.byref(ns), src, dst, w, nw) == 0
        return list(src), list(dst), list(w)

    query()
    assert fill() == ([0, 1], [1, 2], [1.5, 2.5])
    query()
    p.write_text("1 2 7.5\n2 3 8.5\n")  # same sizes, new weights, a later modification time
    st = os.stat(p)
    os.utime(p, ns=(st.st_atime_ns, st.st_mtime_ns + 1_000_000_000))
    assert fill() == ([0, 1], [1, 2], [7.5, 8.5])
    assert fill() == ([0, 1], [1, 2], [7.5, 8.5])  # a fill without a size query parses on its own


@pytest.mark.parametrize("m", [10, 9_000_000])
def test_graph_create_rejects_bad_endpoints(built_lib, m):
    """rmx_graph_create checks every endpoint on the host (several threads for
    large inputs) before any device work: one id outside 0..N-1, anywhere,
    is RMX_ERR_INVALID (no device needed to see it)."""
    from relaxmap_b200 import Graph, RmxError
    n = 1000
    src = (np.arange(m, dtype=np.int64) % n).astype(np.int32)
    dst = ((np.arange(m, dtype=np.int64) + 1) % n).astype(np.int32)
    for pos, arr, val in ((m - 1, dst, n), (m // 2, src, -1)):
        a = arr.copy()
        a[pos] = val
        s, d = (a, dst) if arr is src else (src, a)
        with pytest.raises(RmxError) as e:
            Graph.from_edges(s, d, n=n)
        assert e.value.status == 1 and "outside" in str(e.value)


def test_release_device_cache_without_cached_blocks(built_lib):
    """With no cached arena blocks (as on a host without a device) the release
    makes no device call and succeeds."""
    from relaxmap_b200 import release_device_cache
    release_device_cache()


def test_read_clu(built_lib, tmp_path):
    """rmx_read_clu reads what the .clu writer writes (CRLF, module index + 1
    per node) and LF files; wrong vertex counts and labels outside 1..N are
    RMX_ERR_FORMAT, a missing file RMX_ERR_IO."""
    from relaxmap_b200 import RmxError, read_clu
    part = np.array([3, 0, 0, 4, 3, 1], dtype=np.int32)
    p = tmp_path / "a.clu"
    p.write_bytes(b"*Vertices 6\r\n" + b"".join(b"%d\r\n" % (m + 1) for m in part))
    np.testing.assert_array_equal(read_clu(p, 6), part)
    p.write_bytes(b"*Vertices 6\n" + b"".join(b"%d\n" % (m + 1) for m in part))  # LF, no final newline issue
    np.testing.assert_array_equal(read_clu(p, 6), part)
    cases = {b"*Vertices 5\r\n1\r\n1\r\n1\r\n1\r\n1\r\n": 3,                  # 5 vertices, graph has 6
             b"*Vertices 6\r\n1\r\n2\r\n0\r\n1\r\n1\r\n1\r\n": 3,              # label 0
             b"*Vertices 6\r\n1\r\n2\r\n7\r\n1\r\n1\r\n1\r\n": 3,              # label above N
             b"*Vertices 6\r\n1\r\n2\r\nx\r\n1\r\n1\r\n1\r\n": 3,              # not an integer
             b"*Vertices 6\r\n1\r\n2\r\n3\r\n": 3,                             # labels missing
             b"*Network 6\r\n": 3}
    for body, status in cases.items():
        p.write_bytes(body)
        with pytest.raises(RmxError) as e:
            read_clu(p, 6)
        assert e.value.status == status, body
    with pytest.raises(RmxError) as e:
        read_clu(tmp_path / "none.clu", 6)
    assert e.value.status == 2


def test_read_clu_reference_files(built_lib):
    """The .clu files the reference wrote read back label by label."""
    from relaxmap_b200 import read_clu
    files = sorted(GOLDEN.glob("*.ref.clu"))
    assert files
    for f in files:
        labels = [int(x) for x in f.read_bytes().split(b"\r\n")[1:] if x]
        np.testing.assert_array_equal(read_clu(f, len(labels)), np.array(labels) - 1)


def test_degenerate_files_match_the_oracle(built_lib, oracle_mod, tmp_path):
    """Empty and comment-only edge lists, blank lines only (the stream re-reads
    "" and adds node 0), no final newline (one range and many), and a Pajek
    file without links: the same nodes and links as the oracle."""
    from relaxmap_b200 import parse_file
    O = oracle_mod
    cases = {"empty.txt": b"", "comments.txt": b"# a\n# b\n", "blank.txt": b"\n\n\n",
             "nofinal.txt": b"1 2 0.5\n2 3", "crlf_nofinal.txt": b"1 2\r\n3 1 2.5\r",
             "noarcs.net": b"*Vertices 3\n1 \"a\"\n2 \"b\"\n3 \"c\"\n*Arcs\n",
             "noarcs_nofinal.net": b"*Vertices 2\n1\n2\n*Edges"}
    rng = np.random.default_rng(4)
    big = "\n".join(f"{a} {b} {x!r}" for a, b, x in zip(rng.integers(0, 900, 90000).tolist(),
                                                       rng.integers(0, 900, 90000).tolist(),
                                                       rng.uniform(0, 3, 90000).tolist()))
    cases["big_nofinal.txt"] = big.encode()  # > 1 MB: the multi-range parse, last line unterminated
    for name, body in cases.items():
        p = tmp_path / name
        p.write_bytes(body)
        ld = O.parse_pajek(p) if name.endswith(".net") else O.parse_txt(p)
        for t in (1, 7):
            d = parse_file(p, threads=t)
            assert d["n"] == ld.n, name
            acc = {}
            for a, b, x in zip(d["src"].tolist(), d["dst"].tolist(), d["w"].tolist()):
                acc[(a, b)] = acc.get((a, b), 0.0) + x
            ref = {(a, b): x for a, b, x in zip(ld.src.tolist(), ld.dst.tolist(), ld.w.tolist()) if a != b}
            assert acc == ref, name
    assert len(big) > (1 << 20)
