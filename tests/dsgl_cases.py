"""Seeded corpora for the dsgl pin: vertex counts (all distinct, so that dsgl's
std::sort of the vocabulary has one order; more than 1000 vertices, because
dsgl.hpp:374 asserts on vocabulary index 1000) and walks ended by -1, with a few
hot vertices so that subsampling discards tokens."""
import numpy as np

# name: (vertices, walks, size, window, negative, sample, alpha, iter, seed)
CASES = {
    "d32_decay": (1200, 700, 32, 3, 5, 1e-3, 0.025, 1, 1),
    "d128_iter2": (1100, 60, 128, 10, 5, 1e-3, 0.01, 2, 2),
    "d64_nosample_neg1": (1300, 80, 64, 5, 1, 0.0, 0.025, 1, 3),
    "d96_neg8": (1300, 80, 96, 4, 8, 1e-2, 0.05, 1, 4),
}


def make_case(name: str):
    v, n_walks, size, window, negative, sample, alpha, iterations, seed = CASES[name]
    rng = np.random.default_rng(seed)
    counts = (np.arange(v)[::-1] * 3 + 7).astype(np.int32)
    rng.shuffle(counts)
    counts[:20] *= 400
    toks = []
    for _ in range(n_walks):
        n = int(rng.integers(1, 40))
        walk = np.where(rng.random(n) < 0.3, rng.integers(0, 20, n), rng.integers(0, v, n))
        toks.extend(walk.tolist())
        toks.append(-1)
    corpus = np.array(toks, np.int32)
    return dict(counts=counts, corpus=corpus, size=size, window=window, negative=negative, sample=sample,
                alpha=alpha, iterations=iterations)
