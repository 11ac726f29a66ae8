"""The plain (word2vec.cu) rule on BF16 rows (DG_SGNS_PLAIN_BF16) against the
FP32 kernel-order checker and the FP64 checker.

The BF16 trainer forms exactly the FP32 trainer's pairs (same counts); its rows
differ by the BF16 storage of rows beyond the FP32 masters (stochastic
rounding).  Tolerances, relative Frobenius norm after each call of 10 walks:
against the FP32 checker <= 5e-2 with 16 FP32 master rows and <= 1e-6 when
every row is a master (the same arithmetic in the same order); deterministic
runs repeat bit for bit.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
pytestmark = pytest.mark.gpu


def _tiny():
    import dgoracle
    from distger import graphgen
    rounds, _, _ = dgoracle.load_golden(os.path.join(GOLDEN, "tiny200_ref_walks.npz"))
    edges = graphgen.read_edges(os.path.join(GOLDEN, "tiny200.bin"))
    csr = dgoracle.Csr(edges, 200, undirected=True)
    return rounds, (csr.out_deg + csr.in_deg).astype(np.uint32)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def _make(counts, mode, size, master_rows, deterministic=True, seed=11):
    from distger.sgns import SGNS
    return SGNS(200, counts, size=size, window=5, negative=5, sample=1e-3, alpha=0.025, min_count=0, mode=mode,
                deterministic=deterministic, seed=seed, table_size=1_000_000, master_rows=master_rows)


@pytest.mark.parametrize("size", [64, 128])
@pytest.mark.parametrize("master_rows,tol", [(16, 5e-2), (1 << 30, 1e-6)])
def test_bf16_plain_against_fp32_checker(distger_lib, oracle, size, master_rows, tol):
    rounds, counts = _tiny()
    dev = _make(counts, "plain_bf16", size, master_rows)
    ref = oracle.Sgns(counts, size=size, window=5, negative=5, sample=1e-3, alpha=0.025, min_count=0, seed=11,
                      table_size=1_000_000)
    offs, verts = rounds[0]
    for k in range(0, 60, 10):
        o = offs[k:k + 11] - offs[k]
        v = verts[offs[k]:offs[k + 10]]
        p0, w0 = ref.stats_f32.pairs, ref.stats_f32.words
        info = dev.train_host(o, v)
        ref.train(o, v)
        # same pairs and tokens as the FP32 rule (the checker's counters may accumulate across calls)
        assert info.pairs in (ref.stats_f32.pairs, ref.stats_f32.pairs - p0)
        assert info.words in (ref.stats_f32.words, ref.stats_f32.words - w0)
        rows, _ = dev.embedding()
        assert _rel(rows, ref.syn0_f32) <= tol
        assert _rel(dev.output_rows(), ref.syn1_f32) <= tol
        assert _rel(rows, ref.syn0) <= tol + 2e-3
    dev.close()


def test_bf16_plain_deterministic_repeats(distger_lib):
    rounds, counts = _tiny()
    offs, verts = rounds[0]
    out = []
    for _ in range(2):
        dev = _make(counts, "plain_bf16", 128, 16)
        dev.train_host(offs[:101], verts[:int(offs[100])])
        out.append((dev.embedding()[0], dev.output_rows()))
        dev.close()
    assert np.array_equal(out[0][0].view(np.uint32), out[1][0].view(np.uint32))
    assert np.array_equal(out[0][1].view(np.uint32), out[1][1].view(np.uint32))


def test_bf16_plain_hogwild_round(distger_lib):
    """Hogwild on a 10,000-vertex power-law graph with the 1,000 hottest rows as
    FP32 masters: same pair counts as the FP32 trainer, embeddings of the same
    scale (BF16 rows are written back as the warp's copy, so collisions on cold
    rows are rare here; a 200-row vocabulary with 16 masters would not be)."""
    import distger
    from distger import graphgen
    from distger.sgns import SGNS
    edges = graphgen.chung_lu(10_000, 100_000, 2.2, seed=0)
    eng = distger.WalkEngine(seed=5)
    eng.load_graph(10_000, "", make_undirected=True, edges=edges)
    p = eng.run_round(10_000, 1)
    od, idg = eng.graph.degrees()
    kw = dict(size=128, window=10, negative=5, sample=1e-3, alpha=0.025, min_count=0, seed=3, table_size=1_000_000)
    dev = SGNS(10_000, od + idg, mode="plain_bf16", master_rows=1000, **kw)
    fp32 = SGNS(10_000, od + idg, mode="plain", **kw)
    a = dev.train_paths(p)
    b = fp32.train_paths(p)
    assert (a.words, a.trained, a.pairs) == (b.words, b.trained, b.pairs)
    rows, rows32 = dev.embedding()[0], fp32.embedding()[0]
    out, out32 = dev.output_rows(), fp32.output_rows()
    assert np.isfinite(rows).all() and np.isfinite(out).all()
    # 9,000 BF16 rows under ~4,000 concurrent warps: some cold-row updates are lost
    # (measured ratio 0.88 for the input rows); a lost update never adds mass.
    assert 0.8 < np.linalg.norm(rows) / np.linalg.norm(rows32) < 1.05
    assert 0.8 < np.linalg.norm(out) / np.linalg.norm(out32) < 1.05
    p.close()
    dev.close()
    fp32.close()


def test_bf16_plain_rejects_unsupported(distger_lib):
    from distger import DistgerError
    _, counts = _tiny()
    with pytest.raises(DistgerError):
        _make(counts, "plain_bf16", 32, 16)
