"""Staged rows in the BF16 plain mode (sgns_plain_pipe_kernel with BF16 rows).

A BF16 row is written back as the warp's (copy + update), so staging it widens
the window in which another warp's update is overwritten.  The trainer stages
BF16 rows only when the hottest BF16 row is expected to be held by at most 0.5
pairs in flight (dg_sgns_info.bf_staged); these tests check that gate on a
small and a large vocabulary, and on a 200,000-vertex graph where it is on,
that the staged run trains the sequential run's pairs and stays as close to it
as the unstaged kernel does (two warps: relative Frobenius norm within 3x the
unstaged run's difference, plus 1e-4; full grid: norms within 3 %).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UNSTAGED, STAGED2 = 4, 0   # launch shapes {64, 0, 12, 0}, {64, 0, 12, 2}


@pytest.fixture(scope="module")
def big_round():
    import distger
    from distger import graphgen
    edges = graphgen.chung_lu(200_000, 2_000_000, 2.2, seed=1)
    eng = distger.WalkEngine(seed=5)
    eng.load_graph(200_000, "", make_undirected=True, edges=edges)
    p = eng.run_round(200_000, 1, n_walkers=20_000)
    od, idg = eng.graph.degrees()
    yield p, od + idg
    p.close()


def _sgns(counts, **kw):
    from distger.sgns import SGNS
    return SGNS(counts.size, counts, size=128, window=10, negative=5, sample=1e-3, alpha=0.025, min_count=0,
                seed=3, table_size=1_000_000, mode="plain_bf16", **kw)


def _rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b.astype(np.float64)))


def test_gate(distger_lib, big_round):
    from distger import graphgen
    import distger
    edges = graphgen.chung_lu(10_000, 100_000, 2.2, seed=0)
    eng = distger.WalkEngine(seed=5)
    eng.load_graph(10_000, "", make_undirected=True, edges=edges)
    od, idg = eng.graph.degrees()
    small = _sgns(od + idg, master_rows=1000)
    assert not small.bf_staged          # ~8 holders of its hottest BF16 row
    small.close()
    eng.graph.close()
    _, counts = big_round
    big = _sgns(counts)
    assert big.bf_staged
    big.close()


def _train(p, counts, shape=None, **kw):
    s = _sgns(counts, **kw)
    if shape is not None:
        s.set_shape(shape)
    info = s.train_paths(p)
    out = (info, s.embedding()[0], s.output_rows())
    s.close()
    return out


def test_staged_bf16_two_warps_close_to_sequential(distger_lib, big_round):
    p, counts = big_round
    seq = _train(p, counts, deterministic=True)
    plain = _train(p, counts, shape=UNSTAGED, workers=2)
    pipe = _train(p, counts, shape=STAGED2, workers=2)
    for info in (plain[0], pipe[0]):
        assert (info.words, info.trained, info.pairs) == (seq[0].words, seq[0].trained, seq[0].pairs)
    d_plain = max(_rel(plain[1], seq[1]), _rel(plain[2], seq[2]))
    d_pipe = max(_rel(pipe[1], seq[1]), _rel(pipe[2], seq[2]))
    print(f"bf16 staged: rel diff vs sequential {d_pipe:.3e} (unstaged two-warp run {d_plain:.3e})")
    assert np.isfinite(pipe[1]).all() and np.isfinite(pipe[2]).all()
    assert d_pipe <= 3 * d_plain + 1e-4


def test_staged_bf16_full_grid_same_scale(distger_lib, big_round):
    p, counts = big_round
    plain = _train(p, counts, shape=UNSTAGED)
    pipe = _train(p, counts, shape=STAGED2)
    assert (pipe[0].words, pipe[0].trained, pipe[0].pairs) == (plain[0].words, plain[0].trained, plain[0].pairs)
    for a, b in ((pipe[1], plain[1]), (pipe[2], plain[2])):
        assert np.isfinite(a).all()
        r = np.linalg.norm(a) / np.linalg.norm(b)
        print(f"bf16 staged / unstaged norm ratio {r:.4f}")
        assert 0.97 < r < 1.03
