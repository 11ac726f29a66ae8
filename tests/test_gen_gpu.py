"""Device generator, split, CSR build and AUC against their CPU restatements.

Bit-exact: the generated pairs and edge data, the split (kept edges, positives,
negatives), the CSR (rows sorted by neighbour, thresholds as the host-path CSR
of the same edges), and the walks on it (against the walk checker fed the same
rows).  AUC within 1e-9 of the host scorer on the same embedding.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(20_000, 200_000, 2.2, 0.0, True, 11), (20_000, 200_000, 1.9, 600.0, False, 5)]


@pytest.mark.parametrize("n,m,beta,cap,weighted,seed", CASES)
def test_generator_and_split_bit_exact(distger_lib, oracle, n, m, beta, cap, weighted, seed):
    from distger.synth import EdgeList
    e = EdgeList.chung_lu(n, m, beta, seed=seed, max_degree=cap, weighted=weighted)
    want = oracle.chung_lu_keys(n, m, beta, cap, seed)
    src, dst, data = e.to_numpy()
    got = (src.astype(np.uint64) << np.uint64(32)) | dst.astype(np.uint64)
    assert np.array_equal(got, want)
    assert np.array_equal(data, oracle.edge_data(want, seed, weighted))
    t = e.split(0.1, 9)
    kept, (pu, pv), (nu, nv) = oracle.lp_split(want, n, 0.1, 9)
    s2, d2, _ = e.to_numpy()
    assert np.array_equal((s2.astype(np.uint64) << np.uint64(32)) | d2.astype(np.uint64), kept)
    u, v, lab = t.to_numpy()
    k = pu.size
    assert t.n_pos == k and t.n_neg == k
    assert np.array_equal(u[:k], pu) and np.array_equal(v[:k], pv)
    assert np.array_equal(u[k:], nu) and np.array_equal(v[k:], nv)
    assert np.all(lab[:k] == 1) and np.all(lab[k:] == 0)
    t.close()
    e.close()


def test_device_csr_matches_host_csr(distger_lib):
    import distger
    from distger import graphgen
    from distger.synth import EdgeList
    e = EdgeList.chung_lu(20_000, 200_000, 2.2, seed=4)
    src, dst, data = e.to_numpy()
    g = e.graph()
    dev = g.csr()
    rec = np.empty(src.size, graphgen.EDGE_DTYPE)
    rec["src"], rec["dst"], rec["data"] = src, dst, data
    host = distger.Graph(20_000, edges=rec, make_undirected=True).csr()
    assert np.array_equal(dev["offsets"], host["offsets"])
    assert np.array_equal(dev["out_deg"], host["out_deg"]) and np.array_equal(dev["in_deg"], host["in_deg"])
    off = host["offsets"]
    for v in range(20_000):
        a, b = int(off[v]), int(off[v + 1])
        order = np.argsort(host["nbr"][a:b], kind="stable")
        assert np.array_equal(dev["nbr"][a:b], host["nbr"][a:b][order])
        assert np.array_equal(dev["thresholds"][a:b], host["thresholds"][a:b][order])
    row = np.repeat(np.arange(20_000), np.diff(off).astype(np.int64))
    assert np.all(np.diff(dev["nbr"].astype(np.int64))[np.diff(row) == 0] > 0)


def test_walks_on_device_csr_bit_exact(distger_lib, oracle):
    import distger
    from distger import graphgen
    from distger.synth import EdgeList
    e = EdgeList.chung_lu(5_000, 50_000, 2.2, seed=8)
    src, dst, data = e.to_numpy()
    eng = distger.WalkEngine(seed=21)
    eng.set_init_round(5)
    eng.set_minLength(20)
    eng.graph = e.graph()
    p = eng.run_round(5_000, 2)
    offs, verts = p.to_numpy()
    # The checker's CSR keeps record order: feed it both directions sorted by (src, dst).
    a = np.concatenate([src, dst]).astype(np.uint64)
    b = np.concatenate([dst, src]).astype(np.uint64)
    d = np.concatenate([data, data])
    order = np.argsort((a << np.uint64(32)) | b, kind="stable")
    rec = np.empty(order.size, graphgen.EDGE_DTYPE)
    rec["src"], rec["dst"], rec["data"] = a[order], b[order], d[order]
    csr = oracle.Csr(rec, 5_000, undirected=False)
    want = oracle.walk_ids(csr, np.arange(5_000), 2, seed=21)
    assert np.array_equal(offs, want[0]) and np.array_equal(verts, want[1])
    p.close()


def test_auc_matches_host_scorer(distger_lib):
    from distger import lp
    from distger.sgns import SGNS
    from distger.synth import EdgeList
    e = EdgeList.chung_lu(5_000, 50_000, 2.2, seed=6)
    t = e.split(0.1, 3)
    g = e.graph()
    csr = g.csr()
    for mode in ["plain", "minibatch"]:
        s = SGNS(5_000, csr["out_deg"] + csr["in_deg"], size=64, window=5, negative=5, min_count=0, mode=mode,
                 master_rows=1000, table_size=1_000_000)
        rng = np.random.default_rng(1)
        s.set_rows(rng.normal(size=(s.vocab_size, 64)).astype(np.float32) * 0.2)
        rows, ids = s.embedding()
        emb = lp.embedding_by_vertex(rows, ids, 5_000)
        u, v, lab = t.to_numpy()
        want = lp.evaluate(emb, np.stack([u, v], axis=1).astype(np.int64), lab)
        got = t.auc(s)
        assert got["auc"] == pytest.approx(want["auc"], abs=1e-9)
        assert got["auc_cosine"] == pytest.approx(want["auc_cosine"], abs=1e-9)
        s.close()
