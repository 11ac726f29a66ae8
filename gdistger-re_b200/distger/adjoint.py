"""Explicit (input, output) minibatches from walks, for the adjoint entry points.

`pairs_from_walks` cuts skip-gram pairs out of walks the way word2vec's
skip-gram loop does (word2vec.cu:305-340): each kept token is a centre, its
window shrinks by b = U{0..window-1}, every other token within window - b
positions is a context; the pair's input row is the context, its output row the
centre.  Consecutive pairs form minibatches of `batch` (dsgl's 2*window+1 = 21,
dsgl.hpp:832) that share `negative` negatives drawn from the unigram^0.75 table
(word2vec.cu:537-556).  Seeded with numpy's PCG64.
"""
from __future__ import annotations

import numpy as np


def pairs_from_walks(offsets: np.ndarray, verts: np.ndarray, v2w: np.ndarray, table: np.ndarray, window: int = 10,
                     batch: int = 21, negative: int = 5, n_pairs: int = 200_000, seed: int = 1):
    """Returns (inputs, outputs, negatives) as uint32 vocabulary rows; negatives has
    ceil(n_pairs / batch) * negative entries."""
    rng = np.random.default_rng(seed)
    ins, outs = [], []
    have = 0
    for w in range(offsets.size - 1):
        rows = v2w[verts[offsets[w]:offsets[w + 1]]]
        rows = rows[rows >= 0]
        n = rows.size
        if n < 2:
            continue
        shrink = rng.integers(0, window, size=n)
        for t in range(n):
            span = window - shrink[t]
            lo, hi = max(0, t - span), min(n, t + span + 1)
            ctx = np.concatenate([rows[lo:t], rows[t + 1:hi]])
            ins.append(ctx)
            outs.append(np.full(ctx.size, rows[t], dtype=np.int64))
            have += ctx.size
        if have >= n_pairs:
            break
    inputs = np.concatenate(ins)[:n_pairs].astype(np.uint32)
    outputs = np.concatenate(outs)[:n_pairs].astype(np.uint32)
    n_batches = (inputs.size + batch - 1) // batch
    negatives = table[rng.integers(0, table.size, size=n_batches * negative)].astype(np.uint32)
    return inputs, outputs, negatives
