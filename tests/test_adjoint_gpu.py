"""The hand-written SGNS backward (adjoint) kernel against an FP64 reference
gradient and central finite differences (h = 1e-3), in FP32 rows (plain trainer)
and BF16 storage (minibatch trainer, with FP32 master rows for the hottest words).

Workload: a 50,000-vertex power-law graph (Chung-Lu, exponent 2.2, 500,000
edges), 200,000 (centre, context) pairs cut from its walks, minibatches of 21
pairs sharing 5 negatives from the unigram^0.75 table.  Tolerances: loss within
1e-6 relative of FP64; gradient within 1e-5 relative (Frobenius) of FP64;
finite differences within 1e-4 relative + 1e-6 absolute per coordinate; equal
inputs give bit-identical gradients; the step is rows - alpha * gradient rounded
to nearest in the storage type.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def walks():
    import distger
    from distger import graphgen
    edges = graphgen.chung_lu(**graphgen.CONFIGS["c4_adjoint"])
    g = distger.Graph(50_000, edges=edges, make_undirected=True)
    eng = distger.WalkEngine(seed=3)
    eng.graph = g
    paths = eng.run_round(50_000, 2)
    offs, verts = paths.to_numpy()
    csr = g.csr()
    counts = csr["out_deg"] + csr["in_deg"]
    paths.close()
    g.close()
    return offs, verts, counts


def _trainer(counts, mode, d, seed=5):
    from distger.sgns import SGNS
    s = SGNS(50_000, counts, size=d, window=10, negative=5, sample=1e-3, alpha=0.01, min_count=0, mode=mode,
             seed=seed, table_size=10_000_000, master_rows=4096 if mode == "minibatch" else 0)
    rng = np.random.default_rng(d)
    scale = 0.7 / np.sqrt(d)
    s.set_rows(rng.normal(size=(s.vocab_size, d)).astype(np.float32) * scale,
               rng.normal(size=(s.vocab_size, d)).astype(np.float32) * scale)
    return s


def _pairs(s, offs, verts):
    from distger.adjoint import pairs_from_walks
    t = s.tables()
    return pairs_from_walks(offs, verts, t["v2w"], t["table"], window=10, batch=21, negative=5,
                            n_pairs=200_000, seed=9)


def _bf16_rn(x: np.ndarray) -> np.ndarray:
    u = x.astype(np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


CASES = [("plain", 64), ("plain", 128), ("minibatch", 64), ("minibatch", 128)]


@pytest.mark.parametrize("mode,d", CASES)
def test_gradient_against_fp64_and_finite_differences(distger_lib, oracle, walks, mode, d):
    offs, verts, counts = walks
    s = _trainer(counts, mode, d)
    inputs, outputs, negs = _pairs(s, offs, verts)
    assert inputs.size == 200_000
    loss, gi, go = s.loss_grad(inputs, outputs, negs, batch=21, negative=5)
    v = s.embedding()[0].astype(np.float64)   # the stored values (BF16 rounded where stored in BF16)
    u = s.output_rows().astype(np.float64)
    loss64, gi64, go64 = oracle.sgns_loss_grad(v, u, inputs, outputs, negs, 21, 5)
    assert loss == pytest.approx(loss64, rel=1e-6)
    for g, g64 in [(gi, gi64), (go, go64)]:
        err = np.linalg.norm(g.astype(np.float64) - g64) / np.linalg.norm(g64)
        assert err < 1e-5, err
    # central differences of the FP64 loss, restricted to the terms of the row
    h = 1e-3
    rng = np.random.default_rng(1)
    args = (inputs, outputs, negs, 21, 5)
    for table, rows, g in [(0, v, gi), (1, u, go)]:
        used = np.unique(inputs if table == 0 else np.concatenate([outputs, negs]))
        for row in [int(used[0]), int(used[1])] + [int(x) for x in rng.choice(used, 6)]:
            c = int(rng.integers(d))
            plus, minus = rows.copy(), rows.copy()
            plus[row, c] += h
            minus[row, c] -= h
            if table == 0:
                lp = oracle.sgns_loss_grad(plus, u, *args, grad=False, only=(0, row))[0]
                lm = oracle.sgns_loss_grad(minus, u, *args, grad=False, only=(0, row))[0]
            else:
                lp = oracle.sgns_loss_grad(v, plus, *args, grad=False, only=(1, row))[0]
                lm = oracle.sgns_loss_grad(v, minus, *args, grad=False, only=(1, row))[0]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[row, c]) <= 1e-4 * abs(fd) + 1e-6, (table, row, c, fd, g[row, c])
    s.close()


@pytest.mark.parametrize("mode", ["plain", "minibatch"])
def test_gradient_is_deterministic(distger_lib, walks, mode):
    offs, verts, counts = walks
    s = _trainer(counts, mode, 128)
    inputs, outputs, negs = _pairs(s, offs, verts)
    l1, gi1, go1 = s.loss_grad(inputs, outputs, negs)
    l2, gi2, go2 = s.loss_grad(inputs, outputs, negs)
    assert l1 == l2
    assert np.array_equal(gi1.view(np.uint32), gi2.view(np.uint32))
    assert np.array_equal(go1.view(np.uint32), go2.view(np.uint32))
    s.close()


@pytest.mark.parametrize("mode", ["plain", "minibatch"])
def test_step_applies_minus_alpha_gradient(distger_lib, walks, mode):
    offs, verts, counts = walks
    s = _trainer(counts, mode, 64)
    inputs, outputs, negs = _pairs(s, offs, verts)
    v0, u0 = s.embedding()[0], s.output_rows()
    loss0, gi, go = s.loss_grad(inputs, outputs, negs)
    # a full-batch step over 200,000 pairs: largest coordinate change 1e-3
    alpha = np.float32(1e-3 / max(np.abs(gi).max(), np.abs(go).max()))
    loss_step = s.adjoint_step(inputs, outputs, negs, float(alpha))
    assert loss_step == loss0
    v1, u1 = s.embedding()[0], s.output_rows()
    for before, g, after in [(v0, gi, v1), (u0, go, u1)]:
        want = before - alpha * g   # float32: one rounding per operation
        if mode == "minibatch":
            nm = s.master_rows
            want[nm:] = _bf16_rn(want[nm:])
        assert np.array_equal(after.view(np.uint32), want.view(np.uint32))
    loss1, _, _ = s.loss_grad(inputs, outputs, negs, grad=False)
    assert loss1 < loss0
    s.close()


def test_rejects_bad_pairs(distger_lib, walks):
    from distger import DistgerError
    offs, verts, counts = walks
    s = _trainer(counts, "plain", 64)
    with pytest.raises(DistgerError):
        s.loss_grad(np.array([s.vocab_size], np.uint32), np.array([0], np.uint32), np.zeros(5, np.uint32))
    with pytest.raises(DistgerError):
        s.loss_grad(np.array([0], np.uint32), np.array([0], np.uint32), np.zeros(17, np.uint32), negative=17)
    s.close()
