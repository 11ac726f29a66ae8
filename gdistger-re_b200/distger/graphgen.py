"""Seeded synthetic graphs standing in for the paper's datasets.

The reference reads graphs as packed binary edge records (include/storage.hpp:15-37,
`Edge<real_t>` = {u32 src, u32 dst, f32 data}, 12 bytes, include/type.hpp:67-91),
produced by its gconverter tool (src/tools/gconverter.cpp:45-76).  None of the
paper's datasets ship with the reference, so the workloads use Chung-Lu power-law
graphs with the same vertex/edge counts instead.

Generator (edge-sampling Chung-Lu): expected degrees w_i proportional to
(i + 1) ** (-1 / (beta - 1)), scaled so that sum(w) = 2 E and capped at
`max_degree`; both endpoints of each edge are drawn independently with
probability proportional to w; self-loops and repeated undirected pairs are
dropped; every vertex left without an edge gets one edge to a w-weighted random
vertex (the reference asserts that every vertex has positive degree and was
visited, walk.hpp:709-723); vertex ids are finally permuted so that id order
carries no degree information.  Edge data is uniform on (0, 1] (or 1.0 for the
unweighted configuration).
"""
from __future__ import annotations

import numpy as np

EDGE_DTYPE = np.dtype([("src", "<u4"), ("dst", "<u4"), ("data", "<f4")])


def _expected_degrees(n: int, m: int, beta: float, max_degree: float | None) -> np.ndarray:
    gamma = 1.0 / (beta - 1.0)
    w = (np.arange(n, dtype=np.float64) + 1.0) ** (-gamma)
    w *= (2.0 * m) / w.sum()
    if max_degree is not None:
        # Re-scale the tail after capping so the expected edge count stays 2m.
        for _ in range(8):
            np.minimum(w, max_degree, out=w)
            w *= (2.0 * m) / w.sum()
        np.minimum(w, max_degree, out=w)
    return w


def chung_lu(n: int, m: int, beta: float, seed: int = 0, max_degree: float | None = None,
             weighted: bool = True) -> np.ndarray:
    """Return an undirected edge list (each pair once) as a structured EDGE_DTYPE array."""
    if n < 2 or m < 1:
        raise ValueError("need n >= 2 and m >= 1")
    rng = np.random.default_rng(seed)
    w = _expected_degrees(n, m, beta, max_degree)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    keys = np.empty(0, dtype=np.uint64)
    want = m
    for _ in range(16):
        draw = int(want * 1.15) + 16
        s = np.searchsorted(cdf, rng.random(draw), side="right").astype(np.uint64)
        d = np.searchsorted(cdf, rng.random(draw), side="right").astype(np.uint64)
        np.minimum(s, n - 1, out=s)
        np.minimum(d, n - 1, out=d)
        keep = s != d
        lo = np.minimum(s[keep], d[keep])
        hi = np.maximum(s[keep], d[keep])
        keys = np.unique(np.concatenate([keys, (lo << np.uint64(32)) | hi]))
        if keys.size >= m:
            break
        want = m - keys.size
    if keys.size > m:
        keys = rng.permutation(keys)[:m]
    src = (keys >> np.uint64(32)).astype(np.uint32)
    dst = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    # Give every isolated vertex one edge.
    deg = np.bincount(src, minlength=n) + np.bincount(dst, minlength=n)
    iso = np.flatnonzero(deg == 0).astype(np.uint32)
    if iso.size:
        partner = np.searchsorted(cdf, rng.random(iso.size), side="right").astype(np.uint32)
        np.minimum(partner, n - 1, out=partner)
        clash = partner == iso
        partner[clash] = (partner[clash] + 1) % n
        src = np.concatenate([src, iso])
        dst = np.concatenate([dst, partner])
    perm = rng.permutation(n).astype(np.uint32)
    order = rng.permutation(src.size)
    out = np.empty(src.size, dtype=EDGE_DTYPE)
    out["src"] = perm[src[order]]
    out["dst"] = perm[dst[order]]
    if weighted:
        out["data"] = (1.0 - rng.random(src.size, dtype=np.float32)).astype(np.float32)
    else:
        out["data"] = np.float32(1.0)
    return out


def write_edges(path: str, edges: np.ndarray) -> None:
    """Write packed 12-byte records, the reference's binary graph format."""
    np.ascontiguousarray(edges, dtype=EDGE_DTYPE).tofile(path)


def read_edges(path: str) -> np.ndarray:
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size % EDGE_DTYPE.itemsize:
        raise ValueError(f"{path}: size {raw.size} is not a multiple of {EDGE_DTYPE.itemsize}")
    return raw.view(EDGE_DTYPE)


# Workloads (sizes from the paper's dataset table; generator parameters chosen to
# mimic each graph's degree distribution).
CONFIGS = {
    "c1_small": dict(n=10_000, m=100_000, beta=2.2, seed=0, max_degree=None, weighted=True),
    "c2_youtube": dict(n=1_138_499, m=2_990_443, beta=2.1, seed=0, max_degree=28_000, weighted=True),
    "c3_livejournal": dict(n=2_238_731, m=14_000_000, beta=2.3, seed=0, max_degree=None, weighted=True),
    "c4_adjoint": dict(n=50_000, m=500_000, beta=2.2, seed=0, max_degree=None, weighted=True),
}
