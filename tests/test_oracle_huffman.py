"""word2vec's Huffman coding (CreateBinaryTree, word2vec.cu:684-740), restated in
the oracle (dgo_huffman) and in the library's host code, against the reference's
own function run on the host (oracle/_ref/libref_w2v.so, built from
src/word2vec.cu): every word's code bits and inner-node points, on vocabularies
with skewed, tied and small counts.

The hierarchical-softmax kernel branch itself is not run from the reference on
the GPU: skip_gram_kernel / cbow_kernel read the shared f[0] for their `continue`
test (word2vec.cu:342-346, 443-447) while thread 0 may already write the next
node's f[0] (word2vec.cu:337), a race across a barrier-separated loop; the branch's
arithmetic is the negative-sampling branch's (pinned bit for bit) with its own
cut-offs and gradient, restated in oracle/dg_oracle_w2v.c (hs_path).
"""
import os

import numpy as np
import pytest


def _cases():
    rng = np.random.default_rng(0)
    for n in (2, 3, 5, 17, 300, 4000):
        yield np.sort(rng.zipf(1.5, n).clip(1, 10 ** 9))[::-1]
        yield np.full(n, 7)
        yield np.sort(rng.integers(1, 50, n))[::-1]


def test_restatement_matches_reference_tree(oracle):
    if not os.path.exists(oracle.REF_W2V):
        pytest.skip("oracle/_ref/libref_w2v.so not built (make -C oracle ref REF=<reference tree>)")
    for cn in _cases():
        mine = oracle.huffman(cn)
        ref = oracle.ref_huffman(cn)
        for a, b in zip(mine, ref):
            np.testing.assert_array_equal(a, b)


def test_tree_properties(oracle):
    for cn in _cases():
        off, point, code = oracle.huffman(cn)
        n = cn.size
        assert off[0] == 0 and np.all(np.diff(off) >= 1)
        assert point.min() >= 0 and point.max() <= n - 2
        assert set(np.unique(code)) <= {0, 1}
        # Every path starts at the root, and no two words share a code.
        assert np.all(point[off[:-1]] == n - 2)
        words = {tuple(code[off[a]:off[a + 1]]) for a in range(n)}
        assert len(words) == n
