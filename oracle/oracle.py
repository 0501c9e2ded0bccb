"""Oracle wrappers: the plain-C restatement (librmxoracle.so), the reference
compiled from its own sources (_ref/librmxref.so, when built), and a
pure-Python restatement of the two input loaders.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU legs as the checker; never by the relaxmap_b200 package.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent


def _ref_src() -> Path:
    """The reference sources the oracle recipe compiles: RMX_REFERENCE_DIR if
    set, else the recipe's own REF_DIR (oracle/Makefile)."""
    env = os.environ.get("RMX_REFERENCE_DIR")
    if env:
        return Path(env)
    try:
        r = subprocess.run(["make", "-s", "--no-print-directory", "-C", str(ORACLE_DIR), "refdir"],
                           capture_output=True, text=True, timeout=30)
        return Path(r.stdout.strip()) if r.returncode == 0 and r.stdout.strip() else Path("")
    except (OSError, subprocess.SubprocessError):
        return Path("")


REF_SRC = _ref_src()
ORACLE_SO = ORACLE_DIR / "librmxoracle.so"
REF_SO = ORACLE_DIR / "_ref" / "librmxref.so"
REF_BIN = ORACLE_DIR / "_ref" / "ompRelaxmap"

ALPHA = 0.15
BETA = 1.0 - 0.15

_i32 = np.int32
_i64 = np.int64
_f64 = np.float64


def build(reference: bool = True) -> None:
    """Compile the C restatement, and the reference harness when its sources exist."""
    targets = ["oracle"]
    if reference and (REF_SRC / "Module.cpp").is_file():
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), f"REF_DIR={REF_SRC}", *targets], check=True)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


_LIB = None
_REF = None


def lib():
    global _LIB
    if _LIB is None:
        if not ORACLE_SO.exists():
            build(reference=False)
        L = C.CDLL(str(ORACLE_SO))
        L.rmxo_initiate.restype = C.c_int
        L.rmxo_codelength.restype = C.c_double
        L.rmxo_convert.restype = C.c_int
        L.rmxo_node_sweeps.restype = C.c_double
        L.rmxo_mt_rand.restype = C.c_uint32
        L.rmxo_mt_randint.restype = C.c_uint32
        _LIB = L
    return _LIB


def reflib():
    """The reference harness, or None when it was not built (no reference sources)."""
    global _REF
    if _REF is None and REF_SO.exists():
        R = C.CDLL(str(REF_SO))
        R.rmxref_create.restype = C.c_void_p
        R.rmxref_load_file.restype = C.c_void_p
        for fn in ("rmxref_prepare", "rmxref_codelength", "rmxref_all_log_all", "rmxref_calc_codelength",
                   "rmxref_sum_exit", "rmxref_node_sweeps", "rmxref_partition", "rmxref_tot_node_weights",
                   "rmxref_node_weight"):
            getattr(R, fn).restype = C.c_double
        for fn in ("rmxref_num_links", "rmxref_num_map_edges", "rmxref_sn_num_links"):
            getattr(R, fn).restype = C.c_longlong
        for fn in ("rmxref_nnode", "rmxref_convert", "rmxref_node_name", "rmxref_coarse_tune"):
            getattr(R, fn).restype = C.c_int
        _REF = R
    return _REF


# --------------------------------------------------------------------------
# Graph containers
# --------------------------------------------------------------------------

@dataclass
class Loaded:
    """What a reference loader leaves in Network: N, names, node weights, the
    summed edge map (sorted by (src,dst)) and the total node weight."""
    n: int
    names: list
    node_w: np.ndarray
    tot_w: float
    src: np.ndarray
    dst: np.ndarray
    w: np.ndarray


@dataclass
class Prepared:
    """After OmpRelaxmap.cpp:113-135: CSR of kept links and teleport weights."""
    n: int
    off: np.ndarray
    dst: np.ndarray
    w: np.ndarray
    tw: np.ndarray
    n_self: int = 0
    names: list = field(default_factory=list)


def csc(n: int, off: np.ndarray, dst: np.ndarray, vals: np.ndarray):
    """In-links from CSR: sources ascending per destination (OmpRelaxmap.cpp:158-162)."""
    src = np.repeat(np.arange(n, dtype=_i32), np.diff(off))
    order = np.argsort(dst, kind="stable")
    in_off = np.zeros(n + 1, dtype=_i64)
    np.cumsum(np.bincount(dst, minlength=n), out=in_off[1:])
    return in_off, src[order].astype(_i32), vals[order].astype(_f64)


def prepare(ld: Loaded) -> Prepared:
    """Teleport weights and link list as in OmpRelaxmap.cpp:113-135: weights <= 0
    and self-loops dropped, map order (src, dst ascending) kept."""
    tw = ld.node_w / ld.tot_w
    keep = (ld.w > 0.0) & (ld.src != ld.dst)
    n_self = int(((ld.w > 0.0) & (ld.src == ld.dst)).sum())
    s, d, w = ld.src[keep], ld.dst[keep], ld.w[keep]
    off = np.zeros(ld.n + 1, dtype=_i64)
    np.cumsum(np.bincount(s, minlength=ld.n), out=off[1:])
    return Prepared(ld.n, off, d.astype(_i32), w.astype(_f64), tw.astype(_f64), n_self, ld.names)


def from_edges(n: int, src, dst, w=None, node_w=None) -> Loaded:
    """Loader-equivalent state from raw arrays: duplicates summed in input order."""
    src = np.asarray(src, dtype=_i64)
    dst = np.asarray(dst, dtype=_i64)
    w = np.ones(len(src)) if w is None else np.asarray(w, dtype=_f64)
    acc: dict = {}
    for a, b, x in zip(src.tolist(), dst.tolist(), w.tolist()):
        acc[(a, b)] = acc.get((a, b), 0.0) + x
    keys = sorted(acc)
    nw = np.ones(n) if node_w is None else np.asarray(node_w, dtype=_f64)
    return Loaded(n, [str(i + 1) for i in range(n)], nw, float(nw.sum()) if node_w is not None else float(n),
                  np.array([k[0] for k in keys], dtype=_i64), np.array([k[1] for k in keys], dtype=_i64),
                  np.array([acc[k] for k in keys], dtype=_f64))


# --------------------------------------------------------------------------
# Loader restatement (FileIO.cpp)
# --------------------------------------------------------------------------

_INT_RE = re.compile(rb"^[ \t\n\v\f\r]*([+-]?[0-9]+)")
_FLT_RE = re.compile(rb"^[ \t\n\v\f\r]*([+-]?(?:(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?|inf(?:inity)?|nan))",
                     re.IGNORECASE)


def c_atol(b: bytes) -> int:
    """C atoi/atol: optional sign and the longest digit prefix, else 0."""
    m = _INT_RE.match(b)
    return int(m.group(1)) if m else 0


_HEX_RE = re.compile(rb"^[ \t\n\v\f\r]*([+-]?0[xX](?:[0-9a-fA-F]+\.?[0-9a-fA-F]*|\.[0-9a-fA-F]+)(?:[pP][+-]?[0-9]+)?)")


def c_atof(b: bytes) -> float:
    """C atof (strtod) on the longest valid prefix: a hexadecimal floating
    constant (C99, e.g. 0x1p3; the binary exponent is optional), a decimal,
    inf / infinity or nan; else 0.0. Overflow gives +-inf as strtod does."""
    h = _HEX_RE.match(b)
    if h:
        t = h.group(1).decode()
        try:
            return float.fromhex(t)
        except OverflowError:
            return float("-inf") if t.startswith("-") else float("inf")
    m = _FLT_RE.match(b)
    if not m:
        return 0.0
    return float(m.group(1).decode())


def _lines(path) -> list:
    data = Path(path).read_bytes()
    ls = data.split(b"\n")
    if ls and ls[-1] == b"":
        ls.pop()
    return ls


class _Stream:
    """istringstream >> string: whitespace-separated tokens; a failed read
    leaves the target unchanged and the stream failed."""

    def __init__(self, line: bytes):
        self.toks = line.split()
        self.i = 0

    def read(self, cur: bytes) -> bytes:
        if self.i < len(self.toks):
            self.i += 1
            return self.toks[self.i - 1]
        self.i = len(self.toks) + 1
        return cur


def parse_txt(path) -> Loaded:
    """load_linkList_format_network (FileIO.cpp:177-265): '#' lines skipped,
    'from to [w]' summed per pair in file order, ids renumbered ascending. A
    blank line re-reads the previous token (the stream keeps buf), as the
    reference does."""
    buf = b""
    acc: dict = {}
    nodes = set()
    for line in _lines(path):
        if line[:1] == b"#":
            continue
        ss = _Stream(line)
        buf = ss.read(buf)
        a = c_atol(buf)
        buf = ss.read(buf)
        b = c_atol(buf)
        buf = b""
        buf = ss.read(buf)
        w = 1.0 if buf == b"" else c_atof(buf)
        nodes.add(a)
        nodes.add(b)
        acc[(a, b)] = acc.get((a, b), 0.0) + w
    ids = sorted(nodes)
    ren = {v: i for i, v in enumerate(ids)}
    keys = sorted(acc, key=lambda k: (ren[k[0]], ren[k[1]]))
    n = len(ids)
    return Loaded(n, [str(v) for v in ids], np.ones(n), float(n),
                  np.array([ren[k[0]] for k in keys], dtype=_i64), np.array([ren[k[1]] for k in keys], dtype=_i64),
                  np.array([acc[k] for k in keys], dtype=_f64))


class PajekFormatError(ValueError):
    pass


def parse_pajek(path) -> Loaded:
    """load_pajek_format_network (FileIO.cpp:32-171)."""
    lines = _lines(path)
    li = 0
    buf = b""
    n = 0
    while n == 0:
        if li >= len(lines):
            raise PajekFormatError("the network file is not in Pajek format")
        ss = _Stream(lines[li])
        li += 1
        buf = ss.read(buf)
        if buf in (b"*Vertices", b"*vertices", b"*VERTICES"):
            buf = ss.read(buf)
            n = c_atol(buf)
        else:
            raise PajekFormatError("the network file is not in Pajek format")
    if n < 0:
        raise PajekFormatError("negative vertex count")
    names, nw = [], np.ones(n)
    for i in range(n):
        line = lines[li] if li < len(lines) else b""
        li += 1
        ss = _Stream(line)
        buf = ss.read(buf)
        q0, q1 = line.find(b'"'), line.rfind(b'"')
        if q0 < q1:
            names.append(line[q0 + 1:q1].decode("latin-1"))
            ss = _Stream(line[q1 + 1:])
        else:
            ss = _Stream(line)
            buf = ss.read(buf)
            buf = ss.read(buf)
            names.append(buf.decode("latin-1"))
        buf = b"1"
        buf = ss.read(buf)
        x = c_atof(buf)
        nw[i] = 1.0 if x <= 0.0 else x
    line = lines[li] if li < len(lines) else b""
    li += 1
    ss = _Stream(line)
    buf = ss.read(buf)
    if buf not in (b"*Edges", b"*edges", b"*Arcs", b"*arcs"):
        raise PajekFormatError("Number of nodes not matching")
    acc: dict = {}
    while li < len(lines):
        ss = _Stream(lines[li])
        li += 1
        buf = ss.read(buf)
        a = c_atol(buf) - 1
        buf = ss.read(buf)
        b = c_atol(buf) - 1
        buf = b""
        buf = ss.read(buf)
        w = 1.0 if buf == b"" else c_atof(buf)
        acc[(a, b)] = acc.get((a, b), 0.0) + w
    keys = sorted(acc)
    for a, b in keys:
        if a != b and not (0 <= a < n and 0 <= b < n):
            raise PajekFormatError(f"link ({a + 1},{b + 1}) outside 1..{n}")
    return Loaded(n, names, nw, float(nw.sum()), np.array([k[0] for k in keys], dtype=_i64),
                  np.array([k[1] for k in keys], dtype=_i64), np.array([acc[k] for k in keys], dtype=_f64))


def load(path) -> Prepared:
    p = str(path)
    ld = parse_pajek(p) if p[p.rfind("."):] == ".net" else parse_txt(p)
    return prepare(ld)


# --------------------------------------------------------------------------
# Numeric restatement (librmxoracle.so)
# --------------------------------------------------------------------------

def initiate(g: Prepared) -> dict:
    L = lib()
    n, E = g.n, len(g.dst)
    p, f = np.zeros(n), np.zeros(E)
    dsize, ex = np.zeros(n), np.zeros(n)
    dang = np.zeros(n, dtype=np.uint8)
    L0, all_ = C.c_double(), C.c_double()
    it = L.rmxo_initiate(n, _ptr(g.off), _ptr(g.dst), _ptr(g.w), _ptr(g.tw), _ptr(p), _ptr(f), _ptr(dsize),
                         _ptr(ex), _ptr(dang), C.byref(L0), C.byref(all_))
    in_off, in_src, in_f = csc(n, g.off, g.dst, f)
    return dict(p=p, f=f, dsize=dsize, exit=ex, dangling=dang, L0=L0.value, all_log_all=all_.value, iters=it,
                in_off=in_off, in_src=in_src, in_f=in_f)


def codelength(g: Prepared, st: dict, part) -> float:
    part = np.ascontiguousarray(part, dtype=_i32)
    se = C.c_double()
    return lib().rmxo_codelength(g.n, _ptr(g.off), _ptr(g.dst), _ptr(st["f"]), _ptr(st["p"]), _ptr(g.tw),
                                 _ptr(st["dsize"]), _ptr(part), C.c_double(st["all_log_all"]), C.byref(se))


def convert(n: int, off, dst, f, part) -> dict:
    part = np.ascontiguousarray(part, dtype=_i32)
    E = len(dst)
    snm = np.zeros(n, dtype=_i32)
    oo, od, of = np.zeros(n + 1, dtype=_i64), np.zeros(max(E, 1), dtype=_i32), np.zeros(max(E, 1))
    io, is_, if_ = np.zeros(n + 1, dtype=_i64), np.zeros(max(E, 1), dtype=_i32), np.zeros(max(E, 1))
    nl = C.c_longlong()
    nsn = lib().rmxo_convert(n, _ptr(off), _ptr(dst), _ptr(f), _ptr(part), _ptr(snm), _ptr(oo), _ptr(od),
                             _ptr(of), _ptr(io), _ptr(is_), _ptr(if_), C.byref(nl))
    k = nl.value
    return dict(n_sn=nsn, sn_of_mod=snm, out_off=oo[:nsn + 1], out_dst=od[:k], out_f=of[:k], in_off=io[:nsn + 1],
                in_src=is_[:k], in_f=if_[:k])


def module_stats(n_mod: int, p, tw, dsize, out_off, out_dst, f, mod):
    """Module sums (node order) and exits for a unit assignment mod[]."""
    P = np.zeros(n_mod)
    TW = np.zeros(n_mod)
    D = np.zeros(n_mod)
    OUT = np.zeros(n_mod)
    cnt = np.zeros(n_mod, dtype=_i64)
    np.add.at(P, mod, p)
    np.add.at(TW, mod, tw)
    np.add.at(D, mod, dsize)
    np.add.at(cnt, mod, 1)
    src = np.repeat(np.arange(len(mod)), np.diff(out_off))
    cross = mod[src] != mod[out_dst]
    np.add.at(OUT, mod[src[cross]], f[cross])
    ex = np.where(cnt > 0, ALPHA * (1.0 - TW) * P + BETA * (OUT + (1.0 - TW) * D), 0.0)
    return dict(P=P, TW=TW, D=D, OUT=OUT, count=cnt, exit=ex)


def evaluate(units: dict, mod, ms: dict, sum_exit: float, allow_new=None):
    """Snapshot decisions for every unit (see rmx_oracle.h)."""
    n = len(units["p"])
    mod = np.ascontiguousarray(mod, dtype=_i32)
    bm = np.zeros(n, dtype=_i32)
    bd = np.zeros(n)
    an = None if allow_new is None else np.ascontiguousarray(allow_new, dtype=np.uint8)
    lib().rmxo_evaluate(n, _ptr(units["out_off"]), _ptr(units["out_dst"]), _ptr(units["out_f"]),
                        _ptr(units["in_off"]), _ptr(units["in_src"]), _ptr(units["in_f"]), _ptr(units["p"]),
                        _ptr(units["tw"]), _ptr(units["dsize"]), _ptr(units["exit"]), _ptr(mod),
                        _ptr(ms["exit"]), _ptr(ms["P"]), _ptr(ms["TW"]), _ptr(ms["D"]), C.c_double(sum_exit),
                        _ptr(an) if an is not None else None, _ptr(bm), _ptr(bd))
    return bm, bd


def node_sweeps(g: Prepared, st: dict, seed: int, prior: bool, vthresh: float, threshold: float, max_iter: int):
    part = np.zeros(g.n, dtype=_i32)
    ns = C.c_int()
    L = lib().rmxo_node_sweeps(g.n, _ptr(g.off), _ptr(g.dst), _ptr(st["f"]), _ptr(st["in_off"]),
                               _ptr(st["in_src"]), _ptr(st["in_f"]), _ptr(st["p"]), _ptr(g.tw), _ptr(st["dsize"]),
                               _ptr(st["exit"]), _ptr(st["dangling"]), C.c_double(st["L0"]), C.c_uint32(seed),
                               int(prior), C.c_double(vthresh), C.c_double(threshold), max_iter, _ptr(part),
                               C.byref(ns))
    return L, part, ns.value


# --------------------------------------------------------------------------
# The reference itself (harness over its own sources)
# --------------------------------------------------------------------------

class Ref:
    """A reference Network built from loader-equivalent arrays or a file."""

    def __init__(self, loaded: Loaded | None = None, path=None):
        R = reflib()
        if R is None:
            raise RuntimeError("reference harness not built (oracle/_ref/librmxref.so)")
        self.R = R
        if path is not None:
            p = str(path)
            self.h = R.rmxref_load_file(p.encode(), int(p[p.rfind("."):] == ".net"))
        else:
            ld = loaded
            s = np.ascontiguousarray(ld.src, dtype=_i32)
            d = np.ascontiguousarray(ld.dst, dtype=_i32)
            w = np.ascontiguousarray(ld.w, dtype=_f64)
            nw = np.ascontiguousarray(ld.node_w, dtype=_f64)
            self.h = R.rmxref_create(ld.n, len(s), _ptr(s), _ptr(d), _ptr(w), _ptr(nw))
        self.n = R.rmxref_nnode(C.c_void_p(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            self.R.rmxref_destroy(C.c_void_p(self.h))
            self.h = None

    @property
    def _h(self):
        return C.c_void_p(self.h)

    def map_edges(self):
        k = self.R.rmxref_num_map_edges(self._h)
        s, d, w = np.zeros(k, dtype=_i32), np.zeros(k, dtype=_i32), np.zeros(k)
        self.R.rmxref_get_map_edges(self._h, _ptr(s), _ptr(d), _ptr(w))
        return s, d, w

    def names(self):
        out = []
        buf = C.create_string_buffer(4096)
        for i in range(self.n):
            self.R.rmxref_node_name(self._h, i, buf, 4096)
            out.append(buf.value.decode("latin-1"))
        return out

    def node_weights(self):
        return np.array([self.R.rmxref_node_weight(self._h, i) for i in range(self.n)])

    def prepare(self, threads: int = 1) -> float:
        return self.R.rmxref_prepare(self._h, threads)

    def links(self):
        k = self.R.rmxref_num_links(self._h)
        off, d, f = np.zeros(self.n + 1, dtype=_i64), np.zeros(k, dtype=_i32), np.zeros(k)
        self.R.rmxref_get_links(self._h, _ptr(off), _ptr(d), _ptr(f))
        return off, d, f

    def nodes(self):
        n = self.n
        p, tw, ds, ex, dg = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n, dtype=np.uint8)
        self.R.rmxref_get_nodes(self._h, _ptr(p), _ptr(tw), _ptr(ds), _ptr(ex), _ptr(dg))
        return dict(p=p, tw=tw, dsize=ds, exit=ex, dangling=dg)

    def codelength(self) -> float:
        return self.R.rmxref_codelength(self._h)

    def set_flows(self, f):
        f = np.ascontiguousarray(f, dtype=_f64)
        self.R.rmxref_set_flows(self._h, _ptr(f))

    def set_partition(self, part):
        part = np.ascontiguousarray(part, dtype=_i32)
        self.R.rmxref_set_partition(self._h, _ptr(part))

    def calc_codelength(self) -> float:
        return self.R.rmxref_calc_codelength(self._h)

    def convert(self) -> dict:
        nsn = self.R.rmxref_convert(self._h)
        k = self.R.rmxref_sn_num_links(self._h)
        mi, sz, ex, tw, ds = (np.zeros(nsn, dtype=_i32), np.zeros(nsn), np.zeros(nsn), np.zeros(nsn),
                              np.zeros(nsn))
        nm = np.zeros(nsn, dtype=_i32)
        oo, od, of = np.zeros(nsn + 1, dtype=_i64), np.zeros(k, dtype=_i32), np.zeros(k)
        io, is_, if_ = np.zeros(nsn + 1, dtype=_i64), np.zeros(k, dtype=_i32), np.zeros(k)
        self.R.rmxref_sn_get(self._h, _ptr(mi), _ptr(sz), _ptr(ex), _ptr(tw), _ptr(ds), _ptr(nm), _ptr(oo),
                             _ptr(od), _ptr(of), _ptr(io), _ptr(is_), _ptr(if_))
        return dict(n_sn=nsn, modidx=mi, size=sz, exit=ex, tw=tw, dsize=ds, nmembers=nm, out_off=oo, out_dst=od,
                    out_f=of, in_off=io, in_src=is_, in_f=if_)

    def coarse_tune(self, threads=1, threshold=1e-3, max_iter=10):
        """generate_sub_modules on the installed partition: (#sub-modules, sub-module per node, parent per SN)."""
        sub = np.zeros(self.n, dtype=_i32)
        par = np.zeros(self.n, dtype=_i32)
        k = self.R.rmxref_coarse_tune(self._h, threads, C.c_double(threshold), max_iter, _ptr(sub), _ptr(par))
        return k, sub, par[:k]

    def node_sweeps(self, seed, prior, vthresh, threshold, max_iter):
        part = np.zeros(self.n, dtype=_i32)
        ns = C.c_int()
        L = self.R.rmxref_node_sweeps(self._h, C.c_uint(seed), int(prior), C.c_double(vthresh),
                                      C.c_double(threshold), max_iter, _ptr(part), C.byref(ns))
        return L, part, ns.value

    def partition(self, seed=1, threads=1, threshold=1e-3, vthresh=0.0, max_iter=10, prior=True):
        part = np.zeros(self.n, dtype=_i32)
        Lb, Lc, nm = C.c_double(), C.c_double(), C.c_int()
        steps = np.zeros(64)
        ns = C.c_int()
        t = self.R.rmxref_partition(self._h, C.c_uint(seed), threads, C.c_double(threshold), C.c_double(vthresh),
                                    max_iter, int(prior), _ptr(part), C.byref(Lb), C.byref(Lc), C.byref(nm),
                                    _ptr(steps), 64, C.byref(ns))
        return dict(seconds=t, L_bits=Lb.value, L_computed_bits=Lc.value, n_modules=nm.value, part=part,
                    steps=steps[:min(ns.value, 64)].copy())


def _plogp(x: float) -> float:
    import math
    return x * math.log(x) if x > 0.0 else 0.0


def delta_to(units: dict, mod, ms: dict, sum_exit: float, u: int, m: int) -> float:
    """Code-length change of moving unit u to module m (-2: an empty module)
    against a snapshot, by the formula of Module.cpp:1047-1115 (pure Python,
    for single decisions in tests)."""
    A = int(mod[u])
    oA = iA = om = im = 0.0
    for j in range(units["out_off"][u], units["out_off"][u + 1]):
        t = mod[units["out_dst"][j]]
        if t == A:
            oA += BETA * units["out_f"][j]
        elif t == m:
            om += BETA * units["out_f"][j]
    for j in range(units["in_off"][u], units["in_off"][u + 1]):
        t = mod[units["in_src"][j]]
        if t == A:
            iA += BETA * units["in_f"][j]
        elif t == m:
            im += BETA * units["in_f"][j]
    pu, tu, du, eu = units["p"][u], units["tw"][u], units["dsize"][u], units["exit"][u]
    eA, PA, DA, TWA = ms["exit"][A], ms["P"][A], ms["D"][A], ms["TW"][A]
    oA += (ALPHA * pu + BETA * du) * (TWA - tu)
    iA += (ALPHA * (PA - pu) + BETA * (DA - du)) * tu
    nexA = eA - eu + oA + iA
    if m == -2:
        em = Pm = 0.0
        nexm = eu
    else:
        em, Pm = ms["exit"][m], ms["P"][m]
        om += (ALPHA * pu + BETA * du) * ms["TW"][m]
        im += (ALPHA * Pm + BETA * ms["D"][m]) * tu
        nexm = em + eu - om - im
    nse = sum_exit + nexA + nexm - eA - em
    d_all = _plogp(nse) - _plogp(sum_exit)
    d_exit = _plogp(nexA) + _plogp(nexm) - _plogp(eA) - _plogp(em)
    d_stay = _plogp(nexA + PA - pu) + _plogp(nexm + Pm + pu) - _plogp(eA + PA) - _plogp(em + Pm)
    return d_all - 2.0 * d_exit + d_stay
