"""Pin of the SGNS restatement to the reference's own CUDA kernels.

word2vec.cu's skip_gram_kernel, cbow_kernel and __sgNegReuse, compiled
unmodified for sm_100a (oracle/_ref/libref_w2v.so, with a no-op stand-in for the
missing hnswlib submodule), run one sentence per launch; the restatement's
reference form (dgo_w2v_sentences: the kernels' LCG streams and reduction
orders, the per-pair arithmetic the device kernels share) must give:
  * skip_gram_kernel, cbow_kernel: the same rows bit for bit;
  * __sgNegReuse: the same rows within 2e-6 absolute + 1e-5 relative, because the
    kernel sums a pair's updates with shared-memory atomics in warp arrival
    order and evaluates exp() on the device.  Its reduceInWarp adds, at each
    offset, the value of a fixed source lane instead of the partner's; the test
    shows that the restatement reproduces the kernel only with that reduction
    as written (exact_sum = 0), not with the warp sum.
"""
import os

import numpy as np
import pytest

import w2v_cases as W

pytestmark = pytest.mark.gpu


def _lib_or_skip():
    import dgoracle
    if not os.path.exists(dgoracle.REF_W2V):
        pytest.skip("oracle/_ref/libref_w2v.so not built (make -C oracle ref REF=<reference tree>)")


@pytest.fixture(scope="module")
def exp_tab(oracle):
    return W.exp_table()


@pytest.mark.parametrize("name", [n for n, v in W.CASES.items() if v[0] in (0, 1)])
def test_sg_cbow_bit_exact(name, exp_tab):
    _lib_or_skip()
    c = W.make_case(name)
    table = W.unigram_table(c["counts"])
    r0, r1 = W.run_reference_kernels(c, table, exp_tab)
    m0, m1 = W.run_restatement(c, table, exp_tab)
    assert not np.array_equal(r0, c["syn0"]) and not np.array_equal(r1, c["syn1"])
    assert np.array_equal(r0.view(np.uint32), m0.view(np.uint32))
    assert np.array_equal(r1.view(np.uint32), m1.view(np.uint32))


def test_negreuse_within_tolerance(exp_tab):
    _lib_or_skip()
    c = W.make_case("reuse200")
    table = W.unigram_table(c["counts"])
    r0, r1 = W.run_reference_kernels(c, table, exp_tab)
    m0, m1 = W.run_restatement(c, table, exp_tab, exact_sum=0)
    np.testing.assert_allclose(m0, r0, rtol=1e-5, atol=2e-6)
    np.testing.assert_allclose(m1, r1, rtol=1e-5, atol=2e-6)
    x0, _ = W.run_restatement(c, table, exp_tab, exact_sum=1)
    assert np.abs(x0 - r0).max() > 100 * np.abs(m0 - r0).max() + 1e-3


@pytest.mark.parametrize("name,size", [("tiny200_mc5", 128), ("cl10k_mc0", 128), ("cl10k_mc0", 100)])
def test_vocab_unigram_table_and_initial_rows_match_reference(distger_lib, name, size):
    """The library's vocabulary, unigram table (the reference's 1e8 slots) and
    initial input rows (size 100 stored padded to 128) equal word2vec.cu's own ReadVocabFromDegree + SortVocab,
    InitUnigramTable and InitNet (word2vec.cu:537-556, 791-809, 844-878) run from
    oracle/_ref/libref_w2v.so, bit for bit."""
    import ctypes as C
    import sys

    import dgoracle
    from distger.sgns import SGNS
    _lib_or_skip()
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_vocab_golden as g
    counts = g.case_counts(name)
    min_count = g.CASES[name][4]
    ids, cn, tw = g.ref_vocab(counts, min_count)
    L = C.CDLL(dgoracle.REF_W2V)
    L.ref_w2v_unigram.argtypes = [C.c_void_p]
    L.ref_w2v_init_rows.argtypes = [C.c_int, C.c_void_p]
    table = np.zeros(L.ref_w2v_table_size(), np.int32)
    assert L.ref_w2v_unigram(table.ctypes.data) == 0
    rows_ref = np.zeros((ids.size, size), np.float32)
    assert L.ref_w2v_init_rows(size, rows_ref.ctypes.data) == 0
    s = SGNS(counts.size, counts, size=size, window=5, negative=5, sample=1e-3, min_count=min_count, mode="plain",
             seed=1, table_size=0)
    rows, vids = s.embedding()
    np.testing.assert_array_equal(vids, ids)
    assert s.train_words == tw
    t = s.tables()
    assert t["table"].size == table.size
    np.testing.assert_array_equal(t["table"], table)
    assert np.array_equal(rows.view(np.uint32), rows_ref.view(np.uint32))
    s.close()
