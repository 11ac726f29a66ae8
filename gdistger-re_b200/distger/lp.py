"""Link-prediction split and AUC scoring for the embeddings.

Split: the hold-out rule of the reference's gtrain tool (src/tools/gtrain.cpp:
226-386): `frac * |E|` edges are removed one at a time, each drawn uniformly
from the remaining edges and accepted only while both endpoints keep an
(undirected) degree above 1 in the shrinking graph; the same number of negative
pairs are drawn uniformly among vertex pairs that are neither edges of the full
graph nor already drawn.  Seeded here (gtrain seeds with time(0)).

Score: sigmoid of the dot product of the two vertices' input embeddings
(cosine reported too); AUC as the Mann-Whitney rank statistic with ties
averaged.  The reference ships no scorer; this one is used for every run.
"""
from __future__ import annotations

import numpy as np


def split(edges: np.ndarray, v_num: int, frac: float = 0.1, seed: int = 2):
    """Returns (train_edges, test_pairs int64[n, 2], test_labels int8[n])."""
    rng = np.random.default_rng(seed)
    src = edges["src"].astype(np.int64)
    dst = edges["dst"].astype(np.int64)
    m = src.size
    npos = int(frac * m)
    deg = np.bincount(src, minlength=v_num) + np.bincount(dst, minlength=v_num)
    held = np.zeros(m, dtype=bool)
    order = rng.permutation(m)
    taken = 0
    deg_l = deg.tolist()
    for e in order.tolist():
        if taken == npos:
            break
        s, d = int(src[e]), int(dst[e])
        if deg_l[s] <= 1 or deg_l[d] <= 1:
            continue
        deg_l[s] -= 1
        deg_l[d] -= 1
        held[e] = True
        taken += 1
    pos = np.stack([src[held], dst[held]], axis=1)
    # Negatives: uniform pairs that are not edges (either direction) and not repeated.
    key = lambda a, b: np.minimum(a, b) * v_num + np.maximum(a, b)  # noqa: E731
    existing = set(key(src, dst).tolist())
    chosen = set()
    neg = []
    while len(neg) < taken:
        a = rng.integers(0, v_num, size=2 * (taken - len(neg)) + 16)
        b = rng.integers(0, v_num, size=a.size)
        for x, y in zip(a.tolist(), b.tolist()):
            if x == y:
                continue
            k = min(x, y) * v_num + max(x, y)
            if k in existing or k in chosen:
                continue
            chosen.add(k)
            neg.append((x, y))
            if len(neg) == taken:
                break
    neg = np.array(neg, dtype=np.int64).reshape(-1, 2)
    pairs = np.concatenate([pos, neg])
    labels = np.concatenate([np.ones(len(pos), np.int8), np.zeros(len(neg), np.int8)])
    return edges[~held], pairs, labels


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
