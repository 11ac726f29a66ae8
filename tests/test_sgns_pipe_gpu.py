"""The staged-rows Hogwild kernel (sgns_plain_pipe_kernel, launch shapes with
staged pairs) against the sequential plain kernel.

It forms exactly the sequential kernel's pairs (same word, token and pair
counts).  Its rows differ from the one-warp sequential run by Hogwild effects
only: two warps' concurrent updates (as in any Hogwild run) plus negatives'
rows copied up to S pairs before this warp's own last update of them.  The
bound below states that, after one round of 10,000 walks on a 10,000-vertex
power-law graph, that difference stays within 3x the difference the two-warp
Hogwild run of the unstaged kernel shows (relative Frobenius norm), plus 1e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UNSTAGED, STAGED2, STAGED3 = 4, 0, 10   # launch shapes {64, 0, 12, 0}, {64, 0, 12, 2}, {64, 0, 12, 3}


@pytest.fixture(scope="module")
def round1():
    import distger
    from distger import graphgen
    edges = graphgen.chung_lu(10_000, 100_000, 2.2, seed=0)
    eng = distger.WalkEngine(seed=5)
    eng.load_graph(10_000, "", make_undirected=True, edges=edges)
    p = eng.run_round(10_000, 1)
    od, idg = eng.graph.degrees()
    yield p, od + idg
    p.close()


def _train(p, counts, shape=None, **kw):
    from distger.sgns import SGNS
    s = SGNS(10_000, counts, size=128, window=10, negative=5, sample=1e-3, alpha=0.025, min_count=0, seed=3,
             table_size=1_000_000, **kw)
    if shape is not None:
        s.set_shape(shape)
    info = s.train_paths(p)
    rows, out = s.embedding()[0], s.output_rows()
    s.close()
    return info, rows, out


def _rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b.astype(np.float64)))


@pytest.mark.parametrize("staged", [STAGED2, STAGED3])
def test_staged_two_warps_close_to_sequential(distger_lib, round1, staged):
    p, counts = round1
    seq = _train(p, counts, deterministic=True)
    plain = _train(p, counts, shape=UNSTAGED, workers=2)
    pipe = _train(p, counts, shape=staged, workers=2)
    for info in (plain[0], pipe[0]):
        assert (info.words, info.trained, info.pairs) == (seq[0].words, seq[0].trained, seq[0].pairs)
    d_plain = max(_rel(plain[1], seq[1]), _rel(plain[2], seq[2]))
    d_pipe = max(_rel(pipe[1], seq[1]), _rel(pipe[2], seq[2]))
    print(f"staged shape {staged}: rel diff vs sequential {d_pipe:.3e} (unstaged two-warp run {d_plain:.3e})")
    assert np.isfinite(pipe[1]).all() and np.isfinite(pipe[2]).all()
    assert d_pipe <= 3 * d_plain + 1e-4


def test_staged_full_grid_same_scale(distger_lib, round1):
    p, counts = round1
    plain = _train(p, counts, shape=UNSTAGED)
    pipe = _train(p, counts, shape=STAGED2)
    assert (pipe[0].words, pipe[0].trained, pipe[0].pairs) == (plain[0].words, plain[0].trained, plain[0].pairs)
    for a, b in ((pipe[1], plain[1]), (pipe[2], plain[2])):
        assert np.isfinite(a).all()
        assert 0.97 < np.linalg.norm(a) / np.linalg.norm(b) < 1.03


def test_long_walks_fall_back(distger_lib, round1):
    """Walks longer than the staged kernel's sentence buffer train through the
    unstaged kernel: the same counts as the sequential run."""
    _, counts = round1
    rng = np.random.default_rng(0)
    lens = rng.integers(60, 140, size=200)
    offs = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    verts = rng.integers(0, 10_000, size=int(offs[-1])).astype(np.uint32)
    from distger.sgns import SGNS
    kw = dict(size=128, window=10, negative=5, sample=1e-3, alpha=0.025, min_count=0, seed=3, table_size=1_000_000)
    a = SGNS(10_000, counts, deterministic=True, **kw)
    b = SGNS(10_000, counts, workers=2, **kw)
    b.set_shape(STAGED2)
    ia, ib = a.train_host(offs, verts), b.train_host(offs, verts)
    assert (ia.words, ia.trained, ia.pairs) == (ib.words, ib.trained, ib.pairs)
    assert np.isfinite(b.embedding()[0]).all()
    a.close()
    b.close()


@pytest.mark.parametrize("size,negative,window", [(64, 3, 5), (128, 8, 15), (128, 5, 1)])
def test_staged_other_instances(distger_lib, round1, size, negative, window):
    """The staged kernel's other instances (any negative count <= 8, 64-float
    rows, the widest window it takes, window 1) give the sequential pair counts
    and a two-warp result as close to the sequential one as the unstaged kernel's."""
    from distger.sgns import SGNS
    p, counts = round1

    def run(shape=None, **kw):
        s = SGNS(10_000, counts, size=size, window=window, negative=negative, sample=1e-3, alpha=0.025,
                 min_count=0, seed=3, table_size=1_000_000, **kw)
        if shape is not None:
            s.set_shape(shape)
        info = s.train_paths(p)
        out = (info, s.embedding()[0], s.output_rows())
        s.close()
        return out

    seq = run(deterministic=True)
    plain = run(shape=UNSTAGED, workers=2)
    pipe = run(shape=STAGED2, workers=2)
    for info in (plain[0], pipe[0]):
        assert (info.words, info.trained, info.pairs) == (seq[0].words, seq[0].trained, seq[0].pairs)
    d_plain = max(_rel(plain[1], seq[1]), _rel(plain[2], seq[2]))
    d_pipe = max(_rel(pipe[1], seq[1]), _rel(pipe[2], seq[2]))
    print(f"size {size} negative {negative} window {window}: staged {d_pipe:.3e}, unstaged {d_plain:.3e}")
    assert np.isfinite(pipe[1]).all() and np.isfinite(pipe[2]).all()
    assert d_pipe <= 3 * d_plain + 1e-4


def test_staged_short_and_empty_walks(distger_lib, round1):
    """Walks of 0, 1 and 2 tokens (no pairs, one pair each way) in the staged
    kernel: the same counts as the sequential kernel."""
    from distger.sgns import SGNS
    _, counts = round1
    rng = np.random.default_rng(3)
    lens = rng.choice([0, 1, 2, 3, 25], size=3000)
    offs = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    verts = rng.integers(0, 10_000, size=int(offs[-1])).astype(np.uint32)
    kw = dict(size=128, window=10, negative=5, sample=0, alpha=0.025, min_count=0, seed=3, table_size=1_000_000)
    a = SGNS(10_000, counts, deterministic=True, **kw)
    b = SGNS(10_000, counts, workers=2, **kw)
    b.set_shape(STAGED2)
    ia, ib = a.train_host(offs, verts), b.train_host(offs, verts)
    assert (ia.words, ia.trained, ia.pairs) == (ib.words, ib.trained, ib.pairs)
    assert _rel(b.embedding()[0], a.embedding()[0]) < 0.05
    a.close()
    b.close()
