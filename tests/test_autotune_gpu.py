"""Autotuner: every launch shape gives the same walks; tuning leaves the walk
visit counts and the trainer's rows as they were and keeps a valid shape."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    from distger import graphgen
    return graphgen.chung_lu(10_000, 100_000, 2.2, seed=0)


def _engine(edges, seed=4):
    from distger import WalkEngine
    eng = WalkEngine(device=0, seed=seed)
    eng.set_init_round(5)
    eng.set_minLength(20)
    eng.load_graph(10_000, "", make_undirected=True, edges=edges)
    return eng


def test_walks_identical_under_every_shape(distger_lib, c1):
    from distger._lib import check, lib
    eng = _engine(c1)
    ref = None
    for shape in range(6):
        check(lib().dg_walk_set_shape(eng.graph.handle, shape))
        p = eng.run_round(10_000, 3)
        offs, verts = p.to_numpy()
        p.close()
        if ref is None:
            ref = (offs, verts)
        else:
            assert np.array_equal(offs, ref[0]) and np.array_equal(verts, ref[1]), shape
    with pytest.raises(Exception):
        check(lib().dg_walk_set_shape(eng.graph.handle, 6))


def test_walk_autotune_restores_visits(distger_lib, c1):
    eng = _engine(c1)
    p = eng.run_round(10_000, 1)
    p.close()
    before = eng.graph.visits()
    info = eng.autotune(10_000, 2)
    assert len(info["candidates"]) == 6 and 0 <= info["chosen"] < 6
    assert all(c["ms"] > 0 for c in info["candidates"])
    assert np.array_equal(eng.graph.visits(), before)


def test_sgns_autotune_restores_rows(distger_lib, c1):
    from distger.sgns import SGNS
    eng = _engine(c1)
    csr = eng.graph.csr()
    counts = csr["out_deg"] + csr["in_deg"]
    s = SGNS(10_000, counts, size=128, window=10, negative=5, sample=1e-3, alpha=0.01, min_count=0, seed=3,
             table_size=1_000_000)
    p = eng.run_round(10_000, 1)
    s.train_paths(p)
    rows0, out0 = s.embedding()[0], s.output_rows()
    info = s.autotune(p)
    assert len(info["candidates"]) == 12 and 0 <= info["chosen"] < 12
    assert np.array_equal(s.embedding()[0].view(np.uint32), rows0.view(np.uint32))
    assert np.array_equal(s.output_rows().view(np.uint32), out0.view(np.uint32))
    t = s.train_paths(p)
    assert t.words == int(p.info.footprints)
    p.close()
    s.close()
