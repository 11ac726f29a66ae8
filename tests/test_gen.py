"""Device graph generator and split, CPU side: properties of the restatement
(oracle/dg_oracle_gen.c) that the GPU tests compare the device code against."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def keys(oracle):
    return oracle.chung_lu_keys(5000, 50_000, 2.2, 0, 11)


def test_generator_edges_are_unique_sorted_and_loop_free(keys):
    lo, hi = keys >> np.uint64(32), keys & np.uint64(0xFFFFFFFF)
    assert np.all(lo < hi)
    assert np.all(np.diff(keys.astype(np.float64)) > 0)
    assert 0.7 * 50_000 < keys.size <= 50_000 + 5000


def test_generator_leaves_no_vertex_isolated(keys):
    lo, hi = (keys >> np.uint64(32)).astype(np.int64), (keys & np.uint64(0xFFFFFFFF)).astype(np.int64)
    deg = np.bincount(lo, minlength=5000) + np.bincount(hi, minlength=5000)
    assert deg.min() >= 1


def test_generator_is_power_law_and_seeded(oracle, keys):
    lo, hi = (keys >> np.uint64(32)).astype(np.int64), (keys & np.uint64(0xFFFFFFFF)).astype(np.int64)
    deg = np.sort(np.bincount(lo, minlength=5000) + np.bincount(hi, minlength=5000))[::-1]
    assert deg[0] > 20 * np.median(deg)
    assert np.array_equal(oracle.chung_lu_keys(5000, 50_000, 2.2, 0, 11), keys)
    assert not np.array_equal(oracle.chung_lu_keys(5000, 50_000, 2.2, 0, 12), keys)


def test_generator_caps_degrees(oracle):
    k = oracle.chung_lu_keys(5000, 50_000, 1.9, 200.0, 3)
    lo, hi = (k >> np.uint64(32)).astype(np.int64), (k & np.uint64(0xFFFFFFFF)).astype(np.int64)
    deg = np.bincount(lo, minlength=5000) + np.bincount(hi, minlength=5000)
    assert deg.max() < 2 * 200


def test_edge_data_range(oracle, keys):
    d = oracle.edge_data(keys[:2000], 11, True)
    assert d.min() > 0.0 and d.max() <= 1.0 and d.std() > 0.2
    assert np.all(oracle.edge_data(keys[:10], 11, False) == 1.0)


def test_split_rule(oracle, keys):
    kept, (pu, pv), (nu, nv) = oracle.lp_split(keys, 5000, 0.1, 9)
    full = set(keys.tolist())
    pos = (pu.astype(np.uint64) << np.uint64(32)) | pv.astype(np.uint64)
    assert kept.size + pos.size == keys.size
    assert 0.07 * keys.size < pos.size < 0.11 * keys.size
    assert set(kept.tolist()).isdisjoint(pos.tolist()) and set(pos.tolist()) <= full
    lo, hi = (kept >> np.uint64(32)).astype(np.int64), (kept & np.uint64(0xFFFFFFFF)).astype(np.int64)
    assert (np.bincount(lo, minlength=5000) + np.bincount(hi, minlength=5000)).min() >= 1
    nk = (np.minimum(nu, nv).astype(np.uint64) << np.uint64(32)) | np.maximum(nu, nv).astype(np.uint64)
    assert np.all(nu != nv) and not (set(nk.tolist()) & full)
