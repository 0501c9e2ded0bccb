"""CPU FP64 adjoint of the code length of a fixed partition.

TEST INFRASTRUCTURE ONLY: the checker of rmx_adjoint_forward/backward, imported
by tests/ and never by the relaxmap_b200 package.

The forward model is the reference's, with the teleportation probability t as
a variable (the reference fixes it at 0.15):
  row normalisation w~ = w / rowsum                     Module.cpp:237-247
  stationary flow p = (1-t) W~^T p + (t + (1-t) d.p) tw  Module.cpp:340-469
  exit q_m = t(1-TW)P + (1-t)(OUT + (1-TW)D)             Module.cpp:2966-2990
  L = plogp(sum q) - 2 sum plogp(q) + sum plogp(q+P) - sum plogp(p)
                                                        Module.cpp:2991-3002
Unlike the device path (power iteration, then an iterated transposed solve),
small systems are solved here directly: a sparse LU of I - (1-t) W~^T (resp.
of its transpose) and a Sherman-Morrison correction for the rank-one dangling
term; large ones by the Neumann series with scipy sparse products. Gradients
are checked against centred finite differences of the reference itself
(oracle/_ref) in tests/test_cpu_adjoint.py.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl


def _plogp(x):
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    pos = x > 0
    out[pos] = x[pos] * np.log(x[pos])
    return out


def _log0(x):
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    pos = x > 0
    out[pos] = np.log(x[pos])
    return out


def _solve_rank1(B, u, v, b):
    """x with (I - B - u v^T) x = b, for B sparse with B + u v^T of spectral
    radius below one. Small systems: sparse LU of I - B and a Sherman-Morrison
    correction. Large ones (LU fill-in grows too fast on these graphs): the
    Neumann series x <- b + B x + u (v.x), iterated until the L1 change is below
    1e-16 of the L1 norm."""
    n = B.shape[0]
    if n <= 4000:
        lu = spl.splu((sp.identity(n, format="csc") - B).tocsc())
        y1 = lu.solve(b)
        y2 = lu.solve(u)
        return y1 + y2 * (v @ y1) / (1.0 - v @ y2)
    B = B.tocsr()
    x = b.copy()
    for _ in range(20000):
        xn = b + B @ x + u * (v @ x)
        done = np.abs(xn - x).sum() <= 1e-16 * np.abs(xn).sum()
        x = xn
        if done:
            break
    return x


def _graph(off, dst, w):
    n = len(off) - 1
    src = np.repeat(np.arange(n), np.diff(off))
    rowsum = np.bincount(src, weights=w, minlength=n)
    wt = w / rowsum[src] if len(w) else w
    dang = (np.diff(off) == 0).astype(np.float64)
    return n, src, rowsum, wt, dang


def forward(off, dst, w, tw, part, t: float = 0.15) -> dict:
    """L (nats) of partition part, the stationary flow and the module terms."""
    n, src, rowsum, wt, dang = _graph(off, dst, w)
    b = 1.0 - t
    WT = sp.csr_matrix((wt, (dst, src)), shape=(n, n))  # W~^T
    p = _solve_rank1(b * WT, b * tw, dang, t * tw)
    part = np.asarray(part)
    M = n
    P = np.bincount(part, weights=p, minlength=M)
    TW = np.bincount(part, weights=tw, minlength=M)
    D = np.bincount(part, weights=p * dang, minlength=M)
    cross_links = part[src] != part[dst]
    cross = np.bincount(src[cross_links], weights=wt[cross_links], minlength=n)  # sum of w~ leaving a's module
    OUT = np.bincount(part, weights=p * cross, minlength=M)
    used = np.bincount(part, minlength=M) > 0
    q = np.where(used, t * (1 - TW) * P + b * (OUT + (1 - TW) * D), 0.0)
    Q = q.sum()
    L = float(_plogp(Q) - 2 * _plogp(q).sum() + _plogp(q + P).sum() - _plogp(p).sum())
    return dict(L=L, p=p, P=P, TW=TW, D=D, OUT=OUT, q=q, Q=Q, cross=cross, src=src, rowsum=rowsum, wt=wt,
                dang=dang, used=used)


def backward(off, dst, w, tw, part, t: float = 0.15) -> dict:
    """dL/dw per link (CSR order), dL/dt and L."""
    fw = forward(off, dst, w, tw, part, t)
    n = len(off) - 1
    b = 1.0 - t
    part = np.asarray(part)
    p, P, TW, D, OUT, q, Q = fw["p"], fw["P"], fw["TW"], fw["D"], fw["OUT"], fw["q"], fw["Q"]
    src, rowsum, wt, dang, used = fw["src"], fw["rowsum"], fw["wt"], fw["dang"], fw["used"]
    g = np.where(used, _log0(np.array([Q]))[0] - 2 * _log0(q) + _log0(q + P), 0.0)
    h = np.where(used, _log0(q + P) + 1.0, 0.0)
    gm, hm = g[part], h[part]
    c = gm * (1 - TW[part]) * (t + b * dang) + hm - (_log0(p) + 1.0) + b * gm * fw["cross"]
    # lambda: (I - b W~ - b d tw^T) lambda = c
    W = sp.csr_matrix((wt, (src, dst)), shape=(n, n))
    lam = _solve_rank1(b * W, b * dang, tw, c)
    G = b * p[src] * (np.where(part[src] != part[dst], gm[src], 0.0) + lam[dst])
    r = np.bincount(src, weights=wt * G, minlength=n)
    grad = (G - r[src]) / rowsum[src] if len(w) else np.zeros(0)
    explicit_t = float((g * ((1 - TW) * P - OUT - (1 - TW) * D))[used].sum())
    dt = explicit_t + (lam @ tw - lam @ p) / b
    return dict(L=fw["L"], dL_dw=grad, dL_dt=dt, lam=lam, p=p)
