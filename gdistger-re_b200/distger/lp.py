"""Link-prediction split and AUC scoring for the embeddings.

Split: the reference's gtrain tool (src/tools/gtrain.cpp:226-386) step for
step, with its random stream: the C library's rand() seeded by srand(seed)
(gtrain seeds with time(0); given that seed the split here is the tool's, edge
for edge and in the same order).  npos = (float) frac * |E| edges are removed
one at a time: an index is drawn among the edges not yet removed (get_big_rand)
until both endpoints have an (undirected) degree above 1, the edge is taken,
both degrees drop by one and the edge is swapped with the last one kept.  As
many negative pairs are drawn (source, then destination, each get_big_rand over
the vertices) until the pair is not an edge of the full graph in either
direction and not a pair already drawn in that direction.

Score: sigmoid of the dot product of the two vertices' input embeddings
(cosine reported too); AUC as the Mann-Whitney rank statistic with ties
averaged.  The reference ships no scorer; this one is used for every run.
"""
from __future__ import annotations

import ctypes
import ctypes.util

import numpy as np

RAND_MAX = 2147483647   # the C library's (glibc) RAND_MAX, which gtrain's get_big_rand assumes


def _libc():
    return ctypes.CDLL(ctypes.util.find_library("c") or "libc.so.6")


def _big_rand(rand, rng: int) -> int:
    """gtrain.cpp:214-223 (get_big_rand), including its quirks: for ranges of
    RAND_MAX and more it never returns a value below RAND_MAX."""
    if rng < RAND_MAX:
        return rand() % rng
    rounds, mod = rng // RAND_MAX, rng % RAND_MAX
    t = rand() % rounds + 1
    if t == rounds:
        return t * RAND_MAX + rand() % mod
    return t * RAND_MAX + rand() % RAND_MAX


def split(edges: np.ndarray, v_num: int, frac: float = 0.1, seed: int = 2, max_tries: int = 1 << 26):
    """Returns (train_edges in gtrain's output order, test_pairs int64[n, 2],
    test_labels int8[n]): positives first, in the order drawn, then negatives.
    Raises RuntimeError where gtrain would loop forever (no edge left whose
    endpoints both keep a second edge, or no free vertex pair).  It reseeds the
    process's C-library rand() (srand(seed)), as the tool does."""
    c = _libc()
    c.srand.argtypes = [ctypes.c_uint]
    c.rand.restype = ctypes.c_int
    c.srand(ctypes.c_uint(seed & 0xFFFFFFFF))
    rand = c.rand
    src = edges["src"].astype(np.int64).tolist()
    dst = edges["dst"].astype(np.int64).tolist()
    order = list(range(len(src)))          # edges[] of the tool, permuted by its swaps
    m = len(src)
    npos = int(np.float32(frac) * np.float32(m))   # float * size_t in the tool
    deg = (np.bincount(edges["src"], minlength=v_num) + np.bincount(edges["dst"], minlength=v_num)).tolist()
    pos = []
    tail = m - 1
    tries = 0
    for _ in range(npos):
        ep = _big_rand(rand, tail + 1)
        while deg[src[order[ep]]] <= 1 or deg[dst[order[ep]]] <= 1:
            tries += 1
            if tries > max_tries:
                raise RuntimeError("split: no edge left whose endpoints both keep a second edge")
            ep = _big_rand(rand, tail + 1)
        e = order[ep]
        pos.append((src[e], dst[e]))
        deg[src[e]] -= 1
        deg[dst[e]] -= 1
        order[ep], order[tail] = order[tail], order[ep]
        tail -= 1
    # Negatives (gtrain.cpp:328-342): not an edge of the full graph (its CSR has
    # both directions), not drawn before as the same (source, destination).
    existing = set((a * v_num + b) for a, b in zip(src, dst))
    existing.update(b * v_num + a for a, b in zip(src, dst))
    drawn = set()
    neg = []
    for _ in range(npos):
        while True:
            a = _big_rand(rand, v_num)
            b = _big_rand(rand, v_num)
            k = a * v_num + b
            if k not in existing and k not in drawn:
                break
            tries += 1
            if tries > max_tries:
                raise RuntimeError("split: no free vertex pair left for a negative")
        drawn.add(k)
        neg.append((a, b))
    pairs = np.array(pos + neg, dtype=np.int64).reshape(-1, 2)
    labels = np.concatenate([np.ones(len(pos), np.int8), np.zeros(len(neg), np.int8)])
    return edges[np.array(order[:tail + 1], dtype=np.int64)], pairs, labels


def write_split(train: np.ndarray, pairs: np.ndarray, labels: np.ndarray, lpfile: str, test_edges: str,
                test_labels: str) -> None:
    """Writes split()'s result as gtrain writes it (gtrain.cpp:344-385): the
    train edges as `src dst data` lines (data as an unsigned integer), the test
    pairs as `src dst` lines, the labels one per line."""
    with open(lpfile, "w") as f:
        f.writelines(f"{a} {b} {c}\n" for a, b, c in
                     zip(train["src"].tolist(), train["dst"].tolist(), train["data"].astype(np.int64).tolist()))
    with open(test_edges, "w") as f:
        f.writelines(f"{a} {b}\n" for a, b in pairs.tolist())
    with open(test_labels, "w") as f:
        f.writelines(f"{x}\n" for x in labels.tolist())


def auc(scores: np.ndarray, labels: np.ndarray) -> float:
    """Area under the ROC curve (Mann-Whitney U / (n_pos * n_neg)), ties averaged."""
    scores = np.asarray(scores, dtype=np.float64)
    labels = np.asarray(labels).astype(bool)
    order = np.argsort(scores, kind="mergesort")
    ranks = np.empty(scores.size, dtype=np.float64)
    sorted_scores = scores[order]
    # average ranks over ties
    n = scores.size
    boundaries = np.flatnonzero(np.diff(sorted_scores)) + 1
    starts = np.concatenate([[0], boundaries])
    ends = np.concatenate([boundaries, [n]])
    avg = (starts + ends + 1) / 2.0
    for s, e, r in zip(starts, ends, avg):
        ranks[order[s:e]] = r
    n_pos = int(labels.sum())
    n_neg = n - n_pos
    if n_pos == 0 or n_neg == 0:
        return float("nan")
    return float((ranks[labels].sum() - n_pos * (n_pos + 1) / 2.0) / (n_pos * n_neg))


def embedding_by_vertex(rows: np.ndarray, vocab_ids: np.ndarray, v_num: int) -> np.ndarray:
    """Rows in vertex order; vertices outside the vocabulary get zero rows."""
    out = np.zeros((v_num, rows.shape[1]), dtype=np.float32)
    out[vocab_ids] = rows
    return out


def score_pairs(emb: np.ndarray, pairs: np.ndarray):
    a = emb[pairs[:, 0]]
    b = emb[pairs[:, 1]]
    dot = np.einsum("ij,ij->i", a.astype(np.float64), b.astype(np.float64))
    sig = 1.0 / (1.0 + np.exp(-dot))
    na = np.linalg.norm(a, axis=1)
    nb = np.linalg.norm(b, axis=1)
    cos = dot / np.maximum(na * nb, 1e-30)
    return sig, cos


def evaluate(emb: np.ndarray, pairs: np.ndarray, labels: np.ndarray) -> dict:
    sig, cos = score_pairs(emb, pairs)
    return {"auc": auc(sig, labels), "auc_cosine": auc(cos, labels)}


def read_embedding_text(path: str, v_num: int) -> np.ndarray:
    """Reads the reference's embedding text (word2vec.cu:1357-1362 / dsgl.hpp:1443-1460):
    a "rows dims" header, then per row the vertex id followed by its values."""
    with open(path) as f:
        header = f.readline().split()
        d = int(header[1])
        emb = np.zeros((v_num, d), dtype=np.float32)
        for line in f:
            parts = line.split()
            if len(parts) < d + 1:
                continue
            emb[int(parts[0])] = np.array(parts[1:d + 1], dtype=np.float32)
    return emb
