"""ctypes binding of librelaxmap_b200.so (include/relaxmap_b200.h).

There is no CPU fallback: importing works without a GPU, but every call that
computes raises RmxError when the CUDA library or device is unavailable.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "librelaxmap_b200.so"

RMX_OK = 0
STATUS = {0: "RMX_OK", 1: "RMX_ERR_INVALID", 2: "RMX_ERR_IO", 3: "RMX_ERR_FORMAT", 4: "RMX_ERR_CUDA",
          5: "RMX_ERR_OOM", 6: "RMX_ERR_NO_CONVERGENCE", 7: "RMX_ERR_TIMEOUT", 8: "RMX_ERR_STATE"}
KERNELS = ["spmv", "eval", "commit", "coarsen", "codelen", "other", "adjoint"]

# every symbol include/relaxmap_b200.h declares
EXPORTS = ["rmx_last_error", "rmx_version", "rmx_opts_default", "rmx_graph_create", "rmx_graph_load_file",
           "rmx_parse_file",
           "rmx_graph_destroy", "rmx_graph_info", "rmx_graph_links", "rmx_initiate", "rmx_codelength",
           "rmx_coarsen", "rmx_evaluate_moves", "rmx_coarsen_engine", "rmx_evaluate_sn_moves", "rmx_optimize", "rmx_superstep_codelengths", "rmx_write_outputs",
           "rmx_set_profiling", "rmx_get_profile", "rmx_graph_stream", "rmx_sync", "rmx_cli_main",
           "rmx_steady_state_noalloc", "rmx_noalloc_last_error", "rmx_adjoint_forward", "rmx_adjoint_backward",
           "rmx_batch_create", "rmx_batch_set_wave", "rmx_batch_optimize", "rmx_batch_info", "rmx_batch_destroy",
           "rmx_reset_flow", "rmx_release_device_cache", "rmx_get_tuning", "rmx_set_tuning", "rmx_read_clu"]


class RmxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Opts(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("threads", C.c_int32), ("attempts", C.c_int32), ("threshold", C.c_double),
                ("vthresh", C.c_double), ("max_iter", C.c_int32), ("prior", C.c_int32),
                ("sub_batches", C.c_int32), ("verbose", C.c_int32)]


class KernelStat(C.Structure):
    _fields_ = [("launches", C.c_int64), ("ms", C.c_double), ("bytes", C.c_double)]


class Profile(C.Structure):
    _fields_ = [("k", KernelStat * 7), ("sweeps", C.c_int64), ("supersteps", C.c_int64),
                ("power_iters", C.c_int64), ("total_ms", C.c_double), ("kernel_launches", C.c_int64),
                ("links_evaluated", C.c_int64), ("units_evaluated", C.c_int64), ("adjoint_iters", C.c_int64),
                ("level_ms", C.c_double * 3), ("candidates_evaluated", C.c_int64),
                ("eval_bin_ms", C.c_double * 6), ("eval_bin_launches", C.c_int64 * 6),
                ("eval_bin_links", C.c_int64 * 6), ("eval_bin_bytes", C.c_double * 6)]


EVAL_BINS = ["reg", "warp", "mid", "block", "large", "hub"]


_L = None
_P = C.c_void_p


def lib():
    """Load the library (raises if it was not built)."""
    global _L
    if _L is None:
        if not LIB_PATH.exists():
            raise RmxError(4, f"{LIB_PATH} missing: build it with `python -m relaxmap_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        L.rmx_last_error.restype = C.c_char_p
        L.rmx_noalloc_last_error.restype = C.c_char_p
        L.rmx_version.restype = C.c_char_p
        L.rmx_graph_stream.restype = C.c_void_p
        L.rmx_superstep_codelengths.restype = C.c_int32
        for fn in EXPORTS:
            if fn not in ("rmx_last_error", "rmx_version", "rmx_graph_stream", "rmx_superstep_codelengths",
                          "rmx_opts_default", "rmx_noalloc_last_error"):
                getattr(L, fn).restype = C.c_int
        _L = L
    return _L


def _check(st: int):
    if st != RMX_OK:
        raise RmxError(st, lib().rmx_last_error().decode(errors="replace"))


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


def default_opts(**kw) -> Opts:
    o = Opts()
    lib().rmx_opts_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Graph:
    """A graph resident on the GPU (one rmx_graph handle)."""

    def __init__(self, handle):
        self._h = handle
        n, e, s = C.c_int32(), C.c_int64(), C.c_int64()
        _check(lib().rmx_graph_info(self._h, C.byref(n), C.byref(e), C.byref(s)))
        self.n, self.n_links, self.n_self = n.value, e.value, s.value

    @classmethod
    def from_edges(cls, src, dst, w=None, n: int | None = None, node_w=None) -> "Graph":
        src = np.ascontiguousarray(src, dtype=np.int32)
        dst = np.ascontiguousarray(dst, dtype=np.int32)
        if n is None:
            n = int(max(src.max(initial=-1), dst.max(initial=-1))) + 1
        wa = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        nw = None if node_w is None else np.ascontiguousarray(node_w, dtype=np.float64)
        h = C.c_void_p()
        _check(lib().rmx_graph_create(_p(src), _p(dst), _p(wa), C.c_int64(len(src)), C.c_int32(n), _p(nw),
                                      C.byref(h)))
        return cls(h)

    @classmethod
    def from_host_ptrs(cls, src_ptr: int, dst_ptr: int, w_ptr: int | None, n_edges: int, n: int) -> "Graph":
        """Graph from raw host pointers (e.g. pinned buffers)."""
        h = C.c_void_p()
        _check(lib().rmx_graph_create(C.c_void_p(src_ptr), C.c_void_p(dst_ptr),
                                      C.c_void_p(w_ptr) if w_ptr else None, C.c_int64(n_edges), C.c_int32(n), None,
                                      C.byref(h)))
        return cls(h)

    @classmethod
    def from_file(cls, path, threads: int | None = None) -> "Graph":
        """Load a .net / edge-list file with the reference's rules; `threads`
        host parsing threads (default: every core)."""
        threads = _host_threads(threads)
        h = C.c_void_p()
        _check(lib().rmx_graph_load_file(str(path).encode(), C.c_int32(threads), C.byref(h)))
        return cls(h)

    def close(self):
        if self._h:
            lib().rmx_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- queries
    def links(self):
        off = np.zeros(self.n + 1, dtype=np.int64)
        dst = np.zeros(max(self.n_links, 1), dtype=np.int32)
        w = np.zeros(max(self.n_links, 1))
        tw = np.zeros(self.n)
        _check(lib().rmx_graph_links(self._h, _p(off), _p(dst), _p(w), _p(tw)))
        return off, dst[:self.n_links], w[:self.n_links], tw

    def initiate(self) -> dict:
        n, m = self.n, self.n_links
        p, f, ex = np.zeros(n), np.zeros(max(m, 1)), np.zeros(n)
        dg = np.zeros(n, dtype=np.uint8)
        it, L0 = C.c_int32(), C.c_double()
        _check(lib().rmx_initiate(self._h, _p(p), _p(f), _p(ex), _p(dg), C.byref(it), C.byref(L0)))
        return dict(p=p, f=f[:m], exit=ex, dangling=dg, iters=it.value, L0=L0.value)

    def codelength(self, part) -> float:
        part = np.ascontiguousarray(part, dtype=np.int32)
        L = C.c_double()
        _check(lib().rmx_codelength(self._h, _p(part), C.byref(L)))
        return L.value

    def adjoint_forward(self, part, tau: float = 0.15, want_p: bool = False) -> dict:
        """Code length (nats) of a fixed partition at teleportation probability tau."""
        part = np.ascontiguousarray(part, dtype=np.int32)
        L = C.c_double()
        p = np.zeros(self.n) if want_p else None
        _check(lib().rmx_adjoint_forward(self._h, _p(part), C.c_double(tau), C.byref(L),
                                         _p(p) if p is not None else None))
        out = {"L": L.value}
        if p is not None:
            out["p"] = p
        return out

    def adjoint_backward(self, part, tau: float = 0.15, out=None) -> dict:
        """dL/dw per link (CSR order of links()), dL/dtau and L at a fixed partition.
        out: optional float64 array of n_links entries to receive dL/dw (e.g. a
        view of pinned host memory, which the device copies into fastest)."""
        part = np.ascontiguousarray(part, dtype=np.int32)
        if out is not None:
            if out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"] or len(out) < max(self.n_links, 1):
                raise ValueError("out must be a contiguous float64 array of n_links entries")
            g = out
        else:
            g = np.zeros(max(self.n_links, 1))
        dt, L = C.c_double(), C.c_double()
        _check(lib().rmx_adjoint_backward(self._h, _p(part), C.c_double(tau), _p(g), C.byref(dt), C.byref(L)))
        return {"dL_dw": g[: self.n_links], "dL_dtau": dt.value, "L": L.value}

    def coarsen(self, part) -> dict:
        part = np.ascontiguousarray(part, dtype=np.int32)
        n, m = self.n, max(self.n_links, 1)
        nsn, nl = C.c_int32(), C.c_int64()
        snm = np.zeros(n, dtype=np.int32)
        oo, od, of = np.zeros(n + 1, dtype=np.int64), np.zeros(m, dtype=np.int32), np.zeros(m)
        io, is_, if_ = np.zeros(n + 1, dtype=np.int64), np.zeros(m, dtype=np.int32), np.zeros(m)
        _check(lib().rmx_coarsen(self._h, _p(part), C.byref(nsn), C.byref(nl), _p(snm), _p(oo), _p(od), _p(of),
                                 _p(io), _p(is_), _p(if_)))
        k, s = nl.value, nsn.value
        return dict(n_sn=s, sn_of_mod=snm, out_off=oo[:s + 1], out_dst=od[:k], out_f=of[:k], in_off=io[:s + 1],
                    in_src=is_[:k], in_f=if_[:k])

    def coarsen_engine(self, part, part2=None) -> dict:
        """The optimiser's own coarsening of part (then of part2 over the
        first level's modules): fixed-point link sums (value * 2^62), rows in
        the engine's order."""
        part = np.ascontiguousarray(part, dtype=np.int32)
        p2 = None if part2 is None else np.ascontiguousarray(part2, dtype=np.int32)
        if p2 is not None and len(p2) != self.n:
            raise ValueError("part2 needs one module per module id (n entries)")
        n, m = self.n, max(self.n_links, 1)
        nsn, nl = C.c_int32(), C.c_int64()
        snm = np.zeros(n, dtype=np.int32)
        oo, od, of = np.zeros(n + 1, dtype=np.int64), np.zeros(m, dtype=np.int32), np.zeros(m, dtype=np.int64)
        io, is_, if_ = np.zeros(n + 1, dtype=np.int64), np.zeros(m, dtype=np.int32), np.zeros(m, dtype=np.int64)
        st = np.zeros((n, 4), dtype=np.int64)
        _check(lib().rmx_coarsen_engine(self._h, _p(part), _p(p2), C.byref(nsn), C.byref(nl), _p(snm), _p(oo),
                                        _p(od), _p(of), _p(io), _p(is_), _p(if_), _p(st)))
        k, s = nl.value, nsn.value
        return dict(n_sn=s, sn_of_mod=snm, out_off=oo[:s + 1], out_dst=od[:k], out_fx=of[:k], in_off=io[:s + 1],
                    in_src=is_[:k], in_fx=if_[:k], sn_stat=st[:s])

    def evaluate_sn_moves(self, part, sn_part, allow_new=None):
        """Move decisions of the super-nodes of part placed in modules sn_part."""
        part = np.ascontiguousarray(part, dtype=np.int32)
        sp = np.ascontiguousarray(sn_part, dtype=np.int32)
        an = None if allow_new is None else np.ascontiguousarray(allow_new, dtype=np.uint8)
        bm = np.zeros(len(sp), dtype=np.int32)
        bd = np.zeros(len(sp))
        _check(lib().rmx_evaluate_sn_moves(self._h, _p(part), len(sp), _p(sp), _p(an), _p(bm), _p(bd)))
        return bm, bd

    def evaluate_moves(self, part, allow_new=None):
        part = np.ascontiguousarray(part, dtype=np.int32)
        an = None if allow_new is None else np.ascontiguousarray(allow_new, dtype=np.uint8)
        bm = np.zeros(self.n, dtype=np.int32)
        bd = np.zeros(self.n)
        _check(lib().rmx_evaluate_moves(self._h, _p(part), _p(an), _p(bm), _p(bd)))
        return bm, bd

    def optimize(self, **kw) -> dict:
        o = default_opts(**kw)
        part = np.zeros(self.n, dtype=np.int32)
        L, nm = C.c_double(), C.c_int32()
        _check(lib().rmx_optimize(self._h, C.byref(o), _p(part), C.byref(L), C.byref(nm)))
        steps = np.zeros(256)
        ns = lib().rmx_superstep_codelengths(self._h, _p(steps), 256)
        return dict(part=part, L=L.value, L_bits=L.value / math.log(2.0), n_modules=nm.value,
                    steps_bits=steps[:min(ns, 256)].copy())

    def write_outputs(self, part, L: float, outdir: str, name: str):
        part = np.ascontiguousarray(part, dtype=np.int32)
        _check(lib().rmx_write_outputs(self._h, _p(part), C.c_double(L), str(outdir).encode(), name.encode()))

    def set_profiling(self, on: bool):
        _check(lib().rmx_set_profiling(self._h, int(on)))

    def profile(self) -> dict:
        pr = Profile()
        _check(lib().rmx_get_profile(self._h, C.byref(pr)))
        out = {name: dict(launches=pr.k[i].launches, ms=pr.k[i].ms, bytes=pr.k[i].bytes)
               for i, name in enumerate(KERNELS)}
        out.update(sweeps=pr.sweeps, supersteps=pr.supersteps, power_iters=pr.power_iters, total_ms=pr.total_ms,
                   kernel_launches=pr.kernel_launches, links_evaluated=pr.links_evaluated,
                   units_evaluated=pr.units_evaluated, candidates_evaluated=pr.candidates_evaluated,
                   adjoint_iters=pr.adjoint_iters,
                   level_ms={"nodes": pr.level_ms[0], "super_nodes": pr.level_ms[1], "coarse_tune": pr.level_ms[2]},
                   eval_bins={b: dict(ms=pr.eval_bin_ms[i], launches=pr.eval_bin_launches[i],
                                      links=pr.eval_bin_links[i], bytes=pr.eval_bin_bytes[i])
                              for i, b in enumerate(EVAL_BINS)})
        return out

    def reset_flow(self):
        """The next initiate/optimize recomputes the stationary flow."""
        _check(lib().rmx_reset_flow(self._h))

    def stream_ptr(self) -> int:
        return lib().rmx_graph_stream(self._h) or 0

    def sync(self):
        _check(lib().rmx_sync(self._h))


class Batch:
    """Many graphs optimised together, each `attempts` times (rmx_batch_*).

    graphs: a list of (n_nodes, src, dst, w) with graph-local node ids; w may
    be None. node_w: optional list of per-graph node-weight arrays."""

    def __init__(self, graphs, node_w=None):
        self.sizes = np.array([int(g[0]) for g in graphs], dtype=np.int32)
        ne = np.array([len(g[1]) for g in graphs], dtype=np.int64)
        src = np.ascontiguousarray(np.concatenate([np.asarray(g[1], dtype=np.int32) for g in graphs]))
        dst = np.ascontiguousarray(np.concatenate([np.asarray(g[2], dtype=np.int32) for g in graphs]))
        has_w = any(g[3] is not None for g in graphs)
        w = None
        if has_w:
            w = np.ascontiguousarray(np.concatenate([np.ones(len(g[1])) if g[3] is None else
                                                     np.asarray(g[3], dtype=np.float64) for g in graphs]))
        nw = None if node_w is None else np.ascontiguousarray(np.concatenate(node_w), dtype=np.float64)
        h = C.c_void_p()
        _check(lib().rmx_batch_create(C.c_int32(len(graphs)), _p(self.sizes), _p(ne), _p(src), _p(dst), _p(w),
                                      _p(nw), C.byref(h)))
        self._h = h
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes, dtype=np.int64)])

    def set_wave(self, max_links: int, max_nodes: int):
        _check(lib().rmx_batch_set_wave(self._h, C.c_int64(max_links), C.c_int64(max_nodes)))

    def optimize(self, **kw) -> dict:
        o = default_opts(**kw)
        G = len(self.sizes)
        part = np.zeros(int(self.offsets[-1]), dtype=np.int32)
        L, nm, ba = np.zeros(G), np.zeros(G, dtype=np.int32), np.zeros(G, dtype=np.int32)
        _check(lib().rmx_batch_optimize(self._h, C.byref(o), _p(part), _p(L), _p(nm), _p(ba)))
        return {"part": [part[self.offsets[k]:self.offsets[k + 1]] for k in range(G)], "L": L,
                "L_bits": L / np.log(2.0), "n_modules": nm, "best_attempt": ba}

    def info(self) -> dict:
        g, wv, ins, ms = C.c_int32(), C.c_int32(), C.c_int64(), C.c_double()
        _check(lib().rmx_batch_info(self._h, C.byref(g), C.byref(wv), C.byref(ins), C.byref(ms)))
        return {"graphs": g.value, "waves": wv.value, "instances": ins.value, "device_ms": ms.value}

    def close(self):
        if self._h:
            lib().rmx_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _host_threads(threads: int | None) -> int:
    return max(1, os.cpu_count() or 1) if threads is None else int(threads)


def parse_file(path, threads: int | None = None) -> dict:
    """Host-only parse with the loader rules (no GPU needed); `threads` host
    threads (default: every core)."""
    threads = _host_threads(threads)
    n, m, ns = C.c_int32(), C.c_int64(), C.c_int64()
    _check(lib().rmx_parse_file(str(path).encode(), C.c_int32(threads), C.byref(n), C.byref(m), C.byref(ns), None,
                                None, None, None))
    src = np.zeros(max(m.value, 1), dtype=np.int32)
    dst = np.zeros(max(m.value, 1), dtype=np.int32)
    w = np.zeros(max(m.value, 1))
    nw = np.zeros(max(n.value, 1))
    _check(lib().rmx_parse_file(str(path).encode(), C.c_int32(threads), C.byref(n), C.byref(m), C.byref(ns), _p(src),
                                _p(dst), _p(w), _p(nw)))
    k = m.value
    return dict(n=n.value, src=src[:k], dst=dst[:k], w=w[:k], node_w=nw[:n.value], n_self=ns.value)


def steady_state_noalloc(n_nodes: int, n_links: int, in_off_ptr: int, in_src_ptr: int, in_w_ptr: int,
                         teleport_ptr: int, dangling_ptr: int, p_out_ptr: int, iters_ptr: int = 0,
                         stream_ptr: int = 0) -> None:
    """rmx_steady_state_noalloc on caller-owned device buffers (raw pointers)."""
    st = lib().rmx_steady_state_noalloc(C.c_int32(n_nodes), C.c_int64(n_links), C.c_void_p(in_off_ptr),
                                        C.c_void_p(in_src_ptr or None), C.c_void_p(in_w_ptr or None),
                                        C.c_void_p(teleport_ptr), C.c_void_p(dangling_ptr), C.c_void_p(p_out_ptr),
                                        C.c_void_p(iters_ptr or None), C.c_void_p(stream_ptr or None))
    if st != RMX_OK:
        raise RmxError(st, lib().rmx_noalloc_last_error().decode(errors="replace"))


TUNING_FIELDS = ("eval_mid_grid", "eval_block_grid", "eval_large_grid", "eval_warp_grid", "eval_reg_grid",
                 "warp_max_degree", "mid_max_degree", "block_max_degree", "large_max_degree", "hub_partition_links")


class Tuning(C.Structure):
    _fields_ = [(f, C.c_int32) for f in TUNING_FIELDS]


def get_tuning() -> dict:
    """The process-wide launch shape of move evaluation (rmx_get_tuning): grid
    cap of each degree bin in blocks per SM, and the degree bounds of the bins."""
    t = Tuning()
    _check(lib().rmx_get_tuning(C.byref(t)))
    return {f: getattr(t, f) for f in TUNING_FIELDS}


def set_tuning(**values) -> dict:
    """Change some of the grid caps or bin bounds (rmx_set_tuning); the others
    keep their current values. Returns the new setting."""
    unknown = set(values) - set(TUNING_FIELDS)
    if unknown:
        raise ValueError(f"unknown tuning fields {sorted(unknown)}")
    cur = get_tuning()
    cur.update({k: int(v) for k, v in values.items()})
    t = Tuning(*[cur[f] for f in TUNING_FIELDS])
    _check(lib().rmx_set_tuning(C.byref(t)))
    return cur


def read_clu(path, n: int) -> np.ndarray:
    """The partition saved in a .clu file (rmx_read_clu): module index per node."""
    part = np.zeros(max(int(n), 1), dtype=np.int32)
    _check(lib().rmx_read_clu(str(path).encode(), C.c_int32(n), _p(part)))
    return part[:n]


def release_device_cache():
    """Free the device memory that closed handles left in the library's block
    cache (rmx_release_device_cache)."""
    _check(lib().rmx_release_device_cache())


def cli(argv: list[str]) -> int:
    arr = (C.c_char_p * len(argv))(*[a.encode() for a in argv])
    return lib().rmx_cli_main(len(argv), arr)
