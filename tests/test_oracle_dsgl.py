"""Pin of the minibatch (dsgl) restatement to the reference's own trainer.

dgo_dsgl_ref restates Train_SGNS_MPI's compute thread (include/dsgl.hpp:770-1407,
MKL branch) in the reference's random stream and arithmetic order, with the
minibatch step (mb32_step) that the device kernel's restatement
(dgo_sgns_minibatch_f32, bit-exact against the deterministic device mode) also
uses.  It must reproduce, bit for bit, the rows of the unmodified dsgl trainer
(oracle/_ref/ref_dsgl: one compute thread, naive-GEMM stand-in for
cblas_sgemm): against committed fixtures written by that binary
(tests/golden/make_dsgl_golden.py), and live when the binary is built.
"""
import hashlib
import json
import os
import tempfile

import numpy as np
import pytest

import dsgl_cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dsgl_ref.json")


def _digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _restate(oracle, c, **kw):
    return oracle.dsgl_ref(c["counts"], c["corpus"], c["size"], c["window"], c["negative"], c["sample"],
                           c["alpha"], c["iterations"], **kw)


@pytest.mark.parametrize("name", list(dsgl_cases.CASES))
def test_restatement_matches_reference_fixtures(oracle, name):
    want = json.load(open(GOLDEN))[name]
    c = dsgl_cases.make_case(name)
    ids, wih, woh, alpha = _restate(oracle, c)
    assert _digest(ids) == want["ids"]
    assert np.float32(alpha) == np.float32(want["alpha"])
    assert _digest(wih) == want["wih"]
    assert _digest(woh) == want["woh"]


def test_restatement_matches_live_reference(oracle):
    if not os.path.exists(oracle.REF_DSGL):
        pytest.skip("oracle/_ref/ref_dsgl not built (make -C oracle ref REF=<reference tree>)")
    c = dsgl_cases.make_case("d64_nosample_neg1")
    c["corpus"] = c["corpus"][:900]
    c["corpus"][-1] = -1
    with tempfile.TemporaryDirectory() as tmp:
        r_ids, r_wih, r_woh, r_alpha = oracle.run_ref_dsgl(tmp, c["counts"], c["corpus"], c["size"], c["window"],
                                                           c["negative"], 1e-3, c["alpha"], 1, sync_period=3.0)
    c["sample"] = 1e-3
    ids, wih, woh, alpha = _restate(oracle, c)
    assert np.array_equal(ids, r_ids)
    assert np.array_equal(wih.view(np.uint32), r_wih.view(np.uint32))
    assert np.array_equal(woh.view(np.uint32), r_woh.view(np.uint32))


def test_step_order_changes_rows_by_rounding_only(oracle):
    """The same training in the device kernel's step order (split dot products,
    fused chains) stays within FP32 rounding of the reference's order."""
    c = dsgl_cases.make_case("d128_iter2")
    _, wih, woh, _ = _restate(oracle, c)
    _, wih_d, woh_d, _ = _restate(oracle, c, device_order=True)
    assert not np.array_equal(wih, wih_d)
    for a, b in ((wih, wih_d), (woh, woh_d)):
        rel = np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(a.astype(np.float64))
        assert rel < 1e-5, rel
