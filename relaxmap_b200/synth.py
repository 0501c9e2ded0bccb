"""Seeded synthetic directed graphs with the shapes of the benchmark configs.

planted_partition  LFR-style: power-law out-degrees, power-law community sizes,
                   a fraction mu of each node's links leaving its community.
rmat               Kronecker-style R-MAT (a, b, c, d), self-loops and duplicate
                   pairs removed, vertex ids randomly permuted.
Edge lists come back as (src, dst, w) numpy arrays with node ids 0..n-1; w is
None for unweighted graphs.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class SynthGraph:
    n: int
    src: np.ndarray
    dst: np.ndarray
    w: np.ndarray | None
    community: np.ndarray | None = None
    name: str = ""

    @property
    def m(self) -> int:
        return len(self.src)

    def write_edge_list(self, path):
        """The reference's edge-list format: 'from<TAB>to[<TAB>w]', 1-based ids."""
        with open(path, "w") as f:
            if self.w is None:
                np.savetxt(f, np.stack([self.src + 1, self.dst + 1], 1), fmt="%d", delimiter="\t")
            else:
                for a, b, x in zip(self.src + 1, self.dst + 1, self.w):
                    f.write(f"{a}\t{b}\t{x!r}\n")


def _uniq(a: np.ndarray) -> np.ndarray:
    """Sorted distinct values (sort-based; faster than np.unique's hashing here)."""
    a = np.sort(a, kind="stable")
    if len(a) == 0:
        return a
    keep = np.empty(len(a), dtype=bool)
    keep[0] = True
    np.not_equal(a[1:], a[:-1], out=keep[1:])
    return a[keep]


def _powerlaw_mean(a: float, b: float, g: float) -> float:
    if abs(g - 1.0) < 1e-12:
        return (b - a) / math.log(b / a)
    if abs(g - 2.0) < 1e-12:
        return a * b * math.log(b / a) / (b - a)
    return (g - 1) / (g - 2) * (a ** (2 - g) - b ** (2 - g)) / (a ** (1 - g) - b ** (1 - g))


def _sample_powerlaw(rng, size, a, b, g):
    u = rng.random(size)
    if abs(g - 1.0) < 1e-12:
        return a * (b / a) ** u
    e = 1.0 - g
    return (a ** e + u * (b ** e - a ** e)) ** (1.0 / e)


def powerlaw_degrees(rng, n, mean, kmax, g=2.0):
    """Integer degrees from a power law on [kmin, kmax] with the given mean."""
    lo, hi = 1e-3, float(kmax)
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        if _powerlaw_mean(mid, kmax, g) < mean:
            lo = mid
        else:
            hi = mid
    k = np.rint(_sample_powerlaw(rng, n, lo, kmax, g)).astype(np.int64)
    return np.clip(k, 1, kmax)


def planted_partition(n: int, mean_deg: float, max_deg: int, cmin: int, cmax: int, mu: float, seed: int = 42,
                      weights: str | None = None, deg_exp: float = 2.0, comm_exp: float = 1.0) -> SynthGraph:
    rng = np.random.default_rng(seed)
    sizes = []
    tot = 0
    while tot < n:
        s = int(round(_sample_powerlaw(rng, 1, cmin, cmax, comm_exp)[0]))
        s = min(s, n - tot)
        sizes.append(s)
        tot += s
    if len(sizes) > 1 and sizes[-1] < cmin:
        last = sizes.pop()
        sizes[-1] += last
    sizes = np.array(sizes, dtype=np.int64)
    start = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    members = rng.permutation(n).astype(np.int64)  # community c = members[start[c]:start[c]+sizes[c]]
    comm = np.empty(n, dtype=np.int64)
    comm[members] = np.repeat(np.arange(len(sizes)), sizes)
    deg = powerlaw_degrees(rng, n, mean_deg, max_deg, deg_exp)
    k_in_t = np.minimum(np.rint((1.0 - mu) * deg).astype(np.int64), sizes[comm] - 1)
    k_out_t = deg - np.rint((1.0 - mu) * deg).astype(np.int64)

    def draw(k_in, k_out):
        # links inside the community (no self-links)
        u_in = np.repeat(np.arange(n, dtype=np.int64), k_in)
        c = comm[u_in]
        off = rng.integers(0, sizes[c])
        v_in = members[start[c] + off]
        same = v_in == u_in
        v_in[same] = members[start[c[same]] + (off[same] + 1) % sizes[c[same]]]
        # links leaving the community
        u_out = np.repeat(np.arange(n, dtype=np.int64), k_out)
        v_out = rng.integers(0, n, len(u_out))
        for _ in range(64):
            bad = comm[v_out] == comm[u_out]
            if not bad.any():
                break
            v_out[bad] = rng.integers(0, n, int(bad.sum()))
        keep = comm[v_out] != comm[u_out]
        return np.concatenate([u_in * n + v_in, u_out[keep] * n + v_out[keep]])

    key = _uniq(draw(k_in_t, k_out_t))
    for _ in range(6):  # top up links lost to duplicate pairs
        u = key // n
        intra = comm[u] == comm[key % n]
        have_in = np.bincount(u[intra], minlength=n)
        have_out = np.bincount(u[~intra], minlength=n)
        d_in = np.maximum(k_in_t - have_in, 0)
        d_out = np.maximum(k_out_t - have_out, 0)
        if d_in.sum() + d_out.sum() == 0:
            break
        key = _uniq(np.concatenate([key, draw(d_in, d_out)]))
    src, dst = (key // n).astype(np.int32), (key % n).astype(np.int32)
    w = None
    if weights == "uniform":
        w = rng.uniform(1.0, 10.0, len(src))
    elif weights == "lognormal":
        w = rng.lognormal(0.0, 1.0, len(src))
    return SynthGraph(n, src, dst, w, comm.astype(np.int32), f"planted_n{n}_mu{mu}")


def rmat(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 42,
         chunk: int = 1 << 24) -> SynthGraph:
    """R-MAT edges, self-loops and duplicates removed, ids permuted."""
    rng = np.random.default_rng(seed)
    n = 1 << scale
    m = edge_factor * n
    keys = []
    for s0 in range(0, m, chunk):
        k = min(chunk, m - s0)
        u = np.zeros(k, dtype=np.int64)
        v = np.zeros(k, dtype=np.int64)
        for lvl in range(scale):
            r = rng.random(k)
            bu = r >= a + b
            bv = ((r >= a) & (r < a + b)) | (r >= a + b + c)
            u |= bu.astype(np.int64) << lvl
            v |= bv.astype(np.int64) << lvl
        keep = u != v
        keys.append(_uniq(u[keep] * n + v[keep]))
    key = _uniq(np.concatenate(keys))
    perm = rng.permutation(n).astype(np.int64)
    src = perm[key // n].astype(np.int32)
    dst = perm[key % n].astype(np.int32)
    return SynthGraph(n, src, dst, None, None, f"rmat_s{scale}_ef{edge_factor}")


def rmat_device(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 42,
                chunk: int = 1 << 26) -> SynthGraph:
    """R-MAT as rmat(), drawn on the GPU with torch's generator (for scale >= 22,
    where the host generator takes minutes): the same distribution, a different
    stream of random numbers for the same seed."""
    import torch
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    n = 1 << scale
    m = edge_factor * n
    keys = []
    for s0 in range(0, m, chunk):
        k = min(chunk, m - s0)
        u = torch.zeros(k, dtype=torch.int64, device="cuda")
        v = torch.zeros(k, dtype=torch.int64, device="cuda")
        for lvl in range(scale):
            r = torch.rand(k, generator=gen, device="cuda", dtype=torch.float64)
            bu = r >= a + b
            bv = ((r >= a) & (r < a + b)) | (r >= a + b + c)
            u |= bu.to(torch.int64) << lvl
            v |= bv.to(torch.int64) << lvl
        keep = u != v
        keys.append(torch.unique(u[keep] * n + v[keep]))
        del u, v, keep
    key = torch.unique(torch.cat(keys))
    del keys
    perm = torch.randperm(n, generator=gen, device="cuda")
    src = perm[key // n].to(torch.int32).cpu().numpy()
    dst = perm[key % n].to(torch.int32).cpu().numpy()
    return SynthGraph(n, src, dst, None, None, f"rmat_s{scale}_ef{edge_factor}_device")


# The benchmark configurations (sizes, distributions, seeds).
def config_small(seed: int = 42) -> SynthGraph:
    """N=1000, out-degree power law (2, mean 20, max 50), communities power law
    (1) in [10,50], mu=0.3, unweighted."""
    return planted_partition(1000, 20, 50, 10, 50, 0.3, seed)


def config_mid(seed: int = 42, n: int = 1_000_000) -> SynthGraph:
    """N=1e6, mean out-degree 20 (power law 2, max 1000), communities power law
    in [20,1000], mu=0.4, weights U[1,10]."""
    return planted_partition(n, 20, 1000, 20, 1000, 0.4, seed, weights="uniform")


def config_adjoint(seed: int = 42, n: int = 1_000_000) -> SynthGraph:
    return planted_partition(n, 20, 1000, 20, 1000, 0.3, seed, weights="lognormal")


def batched_graphs(n_graphs: int = 4096, seed: int = 42, n_range=(200, 20000), mu_range=(0.1, 0.6),
                   deg_range=(5, 30)) -> list:
    """The batched workload: graphs with N ~ U[200,20000], mu ~ U[0.1,0.6],
    mean out-degree ~ U[5,30] (power law 2, max 10x the mean), communities
    power law in [10,200]; graph k is generated from seed (seed, k)."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_range[0], n_range[1] + 1, n_graphs)
    mus = rng.uniform(*mu_range, n_graphs)
    degs = rng.uniform(*deg_range, n_graphs)
    return [(int(ns[k]), float(degs[k]), float(mus[k]), int(np.random.SeedSequence([seed, k]).generate_state(1)[0]))
            for k in range(n_graphs)]


def batched_graph(spec) -> SynthGraph:
    """One graph of batched_graphs' list."""
    n, deg, mu, s = spec
    return planted_partition(n, deg, max(2, min(n // 2, int(10 * deg))), 10, 200, mu, s)
