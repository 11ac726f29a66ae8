"""The restatement of word2vec.cu's kernels against fixtures the reference's own
kernels wrote (tests/golden/make_w2v_golden.py: skip_gram_kernel, cbow_kernel and
__sgNegReuse compiled unmodified for sm_100a, one sentence per launch).

skip_gram_kernel and cbow_kernel: the restatement's rows hash to the fixture's
(bit-exact).  __sgNegReuse: rows within 2e-6 absolute + 1e-5 relative (the
kernel adds a pair's updates with shared-memory atomics in warp arrival order
and calls the device exp()); only its reduceInWarp as written (a fixed source
lane per step) reproduces them, not the warp sum.
"""
import json
import os

import numpy as np
import pytest

import w2v_cases as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def exp_tab(oracle):
    return W.exp_table()


@pytest.mark.parametrize("name", [n for n, v in W.CASES.items() if v[0] in (0, 1)])
def test_sg_cbow_match_reference_fixture(name, exp_tab):
    want = json.load(open(os.path.join(GOLDEN, "w2v_ref.json")))[name]
    c = W.make_case(name)
    s0, s1 = W.run_restatement(c, W.unigram_table(c["counts"]), exp_tab)
    assert W.digest(s0) == want["syn0"]
    assert W.digest(s1) == want["syn1"]


def test_negreuse_matches_reference_fixture(exp_tab):
    z = np.load(os.path.join(GOLDEN, "w2v_reuse200.npz"))
    c = W.make_case("reuse200")
    table = W.unigram_table(c["counts"])
    s0, s1 = W.run_restatement(c, table, exp_tab, exact_sum=0)
    np.testing.assert_allclose(s0, z["syn0"], rtol=1e-5, atol=2e-6)
    np.testing.assert_allclose(s1, z["syn1"], rtol=1e-5, atol=2e-6)
    x0, _ = W.run_restatement(c, table, exp_tab, exact_sum=1)
    assert np.abs(x0 - z["syn0"]).max() > 1e-3
