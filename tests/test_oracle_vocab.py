"""Pin of the vocabulary restatement to word2vec.cu's own host code.

ReadVocabFromDegree + SortVocab (word2vec.cu:791-809, 629-659; the C library's
qsort by count) run from the reference compiled unmodified
(oracle/_ref/libref_w2v.so): the restatement's vocabulary (dgoracle.Sgns, which
the device build_vocab matches bit for bit, tests/test_sgns_gpu.py) has the same
words in the same order -- ties of equal degree included, thousands of them
here -- the same size after the min_count cut and the same train_words.
Checked against digests of the reference's output (tests/golden/w2v_vocab_ref.json,
tests/golden/make_vocab_golden.py) and, where the library is built, live.
"""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _g():
    sys.path.insert(0, GOLDEN)
    import make_vocab_golden
    return make_vocab_golden


@pytest.mark.parametrize("name", ["tiny200_mc0", "tiny200_mc5", "cl10k_mc0", "cl10k_mc5"])
def test_vocab_matches_reference_golden(oracle, name):
    g = _g()
    with open(os.path.join(GOLDEN, "w2v_vocab_ref.json")) as f:
        ref = json.load(f)[name]
    counts = g.case_counts(name)
    o = oracle.Sgns(counts, size=64, min_count=g.CASES[name][4], table_size=1000)
    ids = np.ascontiguousarray(o.vocab_ids, dtype=np.uint32)
    assert ids.size == ref["vocab_size"]
    assert int(counts[ids].astype(np.int64).sum()) == ref["train_words"]
    assert hashlib.sha256(ids.tobytes()).hexdigest() == ref["ids_sha256"]


@pytest.mark.parametrize("name", ["tiny200_mc5", "cl10k_mc0"])
def test_vocab_matches_reference_live(oracle, name):
    g = _g()
    if not os.path.exists(oracle.REF_W2V):
        pytest.skip("oracle/_ref/libref_w2v.so not built (make -C oracle ref REF=<reference tree>)")
    counts = g.case_counts(name)
    ids, cn, tw = g.ref_vocab(counts, g.CASES[name][4])
    o = oracle.Sgns(counts, size=64, min_count=g.CASES[name][4], table_size=1000)
    np.testing.assert_array_equal(np.asarray(o.vocab_ids, dtype=np.uint32), ids)
    np.testing.assert_array_equal(counts[ids].astype(np.int64), cn)
    assert int(cn.sum()) == tw
