"""Link-prediction split and AUC scorer (CPU).

The split is src/tools/gtrain.cpp:226-386 with the tool's random stream: given
the seed that the tool takes from time(0), its three output files are
reproduced byte for byte -- against digests of the unmodified tool's output
(tests/golden/gtrain_ref.json, tests/golden/make_gtrain_golden.py) and, where
oracle/_ref holds the tool, against a live run of it.  The AUC is checked
against scikit-learn's roc_auc_score, ties included.
"""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GTRAIN = os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "gtrain_ref")


def _golden_cases():
    sys.path.insert(0, GOLDEN)
    import make_gtrain_golden
    return make_gtrain_golden


def _split_files(edges, v, frac, seed):
    """lp.split's result as lp.write_split writes it (the tool's three output formats)."""
    import tempfile

    from distger import lp
    train, pairs, labels = lp.split(edges, v, frac=frac, seed=seed)
    with tempfile.TemporaryDirectory() as d:
        paths = [os.path.join(d, x) for x in ("lp.txt", "te.txt", "tl.txt")]
        lp.write_split(train, pairs, labels, *paths)
        return [open(p, "rb").read() for p in paths]


@pytest.mark.parametrize("name", ["small", "mid", "dense_holdout"])
def test_split_reproduces_gtrain_golden(name):
    g = _golden_cases()
    with open(os.path.join(GOLDEN, "gtrain_ref.json")) as f:
        ref = json.load(f)[name]
    n, _, _, seed, frac = g.CASES[name]
    files = _split_files(g.case_edges(name), n, frac, seed)
    assert [f.count(b"\n") for f in files] == ref["lines"]
    assert [hashlib.sha256(f).hexdigest() for f in files] == ref["sha256"]


@pytest.mark.skipif(not os.path.exists(GTRAIN), reason="reference gtrain not built here (make -C oracle ref)")
@pytest.mark.parametrize("name", ["small", "dense_holdout"])
def test_split_reproduces_gtrain_live(name, tmp_path):
    g = _golden_cases()
    n, _, _, seed, frac = g.CASES[name]
    want = g.run_ref(name, str(tmp_path))
    assert _split_files(g.case_edges(name), n, frac, seed) == want


def test_auc_matches_sklearn():
    from sklearn.metrics import roc_auc_score
    from distger import lp
    rng = np.random.default_rng(0)
    for n, tie_levels in [(50, None), (1000, 7), (5000, None)]:
        labels = rng.integers(0, 2, n).astype(np.int8)
        scores = rng.normal(size=n) + 0.7 * labels
        if tie_levels:
            scores = np.round(scores * tie_levels) / tie_levels
        assert lp.auc(scores, labels) == pytest.approx(roc_auc_score(labels, scores), abs=1e-12)


def test_auc_extremes():
    from distger import lp
    assert lp.auc(np.array([0.1, 0.2, 0.8, 0.9]), np.array([0, 0, 1, 1])) == 1.0
    assert lp.auc(np.array([0.9, 0.8, 0.2, 0.1]), np.array([0, 0, 1, 1])) == 0.0
    assert lp.auc(np.ones(6), np.array([0, 1, 0, 1, 0, 1])) == 0.5
    assert np.isnan(lp.auc(np.ones(3), np.ones(3)))


@pytest.fixture(scope="module")
def c1_split():
    from distger import graphgen, lp
    cfg = graphgen.CONFIGS["c1_small"]
    edges = graphgen.chung_lu(**cfg)
    return cfg["n"], edges, lp.split(edges, cfg["n"], frac=0.1, seed=2)


def test_split_holds_out_ten_percent(c1_split):
    v, edges, (train, pairs, labels) = c1_split
    npos = int(labels.sum())
    assert npos == int(0.1 * edges.size)
    assert labels.size == 2 * npos
    assert train.size == edges.size - npos
    assert np.all(labels[:npos] == 1) and np.all(labels[npos:] == 0)


def test_split_keeps_every_vertex_connected(c1_split):
    v, edges, (train, pairs, labels) = c1_split
    deg = np.bincount(train["src"], minlength=v) + np.bincount(train["dst"], minlength=v)
    full = np.bincount(edges["src"], minlength=v) + np.bincount(edges["dst"], minlength=v)
    # gtrain only removes an edge while both endpoints keep degree > 1 (gtrain.cpp:336-355).
    assert np.all(deg[full > 0] >= 1)


def test_split_positives_are_edges_and_negatives_are_not(c1_split):
    v, edges, (train, pairs, labels) = c1_split
    key = lambda a, b: np.minimum(a, b).astype(np.int64) * v + np.maximum(a, b)  # noqa: E731
    all_keys = set(key(edges["src"], edges["dst"]).tolist())
    train_keys = set(key(train["src"], train["dst"]).tolist())
    pk = key(pairs[:, 0], pairs[:, 1])
    npos = int(labels.sum())
    assert all(k in all_keys and k not in train_keys for k in pk[:npos].tolist())
    neg = pk[npos:].tolist()
    assert not any(k in all_keys for k in neg)
    # gtrain rejects a pair drawn before in the same direction only (gtrain.cpp:202-211).
    directed = (pairs[npos:, 0] * v + pairs[npos:, 1]).tolist()
    assert len(set(directed)) == len(directed)


def test_split_is_seeded(c1_split):
    from distger import lp
    v, edges, (train, pairs, labels) = c1_split
    _, pairs2, _ = lp.split(edges, v, frac=0.1, seed=2)
    np.testing.assert_array_equal(pairs, pairs2)


def test_embedding_text_round_trip(tmp_path):
    from distger import lp
    rng = np.random.default_rng(3)
    emb = rng.normal(size=(5, 4)).astype(np.float32)
    path = tmp_path / "emb.txt"
    with open(path, "w") as f:
        f.write("3 4\n")
        for v in (4, 0, 2):
            f.write("%u " % v + "".join("%lf " % x for x in emb[v]) + "\n")
    got = lp.read_embedding_text(str(path), 5)
    np.testing.assert_allclose(got[[4, 0, 2]], emb[[4, 0, 2]], atol=1e-6)
    assert not got[[1, 3]].any()
