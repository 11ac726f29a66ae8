"""Walk rounds reuse the arena of freed walks (and their per-round counters):
walks of a round are the same whether its arena is fresh, reused from a larger
freed round, or replaced by a bigger allocation; and host-walk training reuses
its staging buffers across calls of different sizes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _engine(edges, max_len=64):
    import distger
    eng = distger.WalkEngine(seed=9, max_len=max_len)
    eng.load_graph(10_000, "", make_undirected=True, edges=edges)
    return eng


@pytest.fixture(scope="module")
def c1():
    from distger import graphgen
    return graphgen.chung_lu(10_000, 100_000, 2.2, seed=0)


def _walks(eng, rnd, n):
    p = eng.run_round(10_000, rnd, n_walkers=n)
    out = p.to_numpy()
    p.close()
    return out


def test_rounds_reusing_arena_match_fresh_rounds(distger_lib, c1):
    reused = _engine(c1)
    sizes = [(2, 500), (3, 10_000), (4, 700), (5, 10_000), (6, 20_000), (7, 300)]
    got = {r: _walks(reused, r, n) for r, n in sizes}
    reused.graph.close()
    for r, n in sizes:
        fresh = _engine(c1)
        ref = _walks(fresh, r, n)
        fresh.graph.close()
        assert np.array_equal(got[r][0], ref[0]) and np.array_equal(got[r][1], ref[1]), (r, n)


def test_host_training_staging_reuse(distger_lib, c1):
    """Deterministic training of the same walks from device paths and from host
    buffers (staging reused across calls that shrink and grow) is bit-identical."""
    from distger.sgns import SGNS
    eng = _engine(c1)
    od, idg = eng.graph.degrees()
    kw = dict(size=128, window=10, negative=5, sample=1e-3, alpha=0.025, min_count=0, seed=3,
              table_size=1_000_000, deterministic=True)
    dev, host = SGNS(10_000, od + idg, **kw), SGNS(10_000, od + idg, **kw)
    for r, n in [(2, 3_000), (3, 200), (4, 5_000)]:
        p = eng.run_round(10_000, r, n_walkers=n)
        offs, verts = p.to_numpy()
        ia = dev.train_paths(p)
        p.close()
        ib = host.train_host(offs, verts)
        assert (ia.words, ia.trained, ia.pairs) == (ib.words, ib.trained, ib.pairs)
    assert np.array_equal(dev.embedding()[0].view(np.uint32), host.embedding()[0].view(np.uint32))
    assert np.array_equal(dev.output_rows().view(np.uint32), host.output_rows().view(np.uint32))
    dev.close()
    host.close()
    eng.graph.close()


def test_host_training_rejects_bad_vertices(distger_lib, c1):
    """A vertex id >= v_num is DG_ERR_ARG (found on the device after the copy) and
    trains nothing; the trainer stays usable."""
    from distger import DistgerError
    from distger.sgns import SGNS
    counts = np.ones(10_000, np.uint32)
    s = SGNS(10_000, counts, size=128, window=5, negative=5, sample=0, alpha=0.025, min_count=0, seed=3,
             table_size=100_000, deterministic=True)
    rows0 = s.embedding()[0].copy()
    offs = np.array([0, 3, 6], np.uint64)
    with pytest.raises(DistgerError):
        s.train_host(offs, np.array([1, 2, 3, 4, 10_000, 5], np.uint32))
    assert np.array_equal(s.embedding()[0].view(np.uint32), rows0.view(np.uint32))
    info = s.train_host(offs, np.array([1, 2, 3, 4, 9_999, 5], np.uint32))
    assert info.words == 6
    s.close()
