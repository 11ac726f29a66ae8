"""Walk kernel parity: the CUDA path (through the C ABI) against the CPU checker.

Bit-exact: CSR, per-entry acceptance thresholds, every walk of every round, the
walk files; FP64 relative entropy within 1e-9 relative (device vs host summation
order).  At full YouTube-shaped size: sampled walker ids checked exactly plus
size-independent properties.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
pytestmark = pytest.mark.gpu


def _golden_edges(name):
    from distger import graphgen
    return graphgen.read_edges(os.path.join(GOLDEN, f"{name}.bin"))


def _engine(edges, v_num, undirected=True, seed=0, max_len=64, min_r=5):
    from distger import WalkEngine
    eng = WalkEngine(device=0, seed=seed, max_len=max_len)
    eng.set_init_round(min_r)
    eng.set_minLength(20)
    eng.load_graph(v_num, "", make_undirected=undirected, edges=edges)
    return eng


@pytest.fixture(scope="module")
def c1_edges():
    from distger import graphgen
    return graphgen.chung_lu(10_000, 100_000, 2.2, seed=0)


@pytest.mark.parametrize("name,v_num", [("tiny200", 200), ("special60", 60)])
def test_csr_and_thresholds_bit_exact(distger_lib, oracle, name, v_num):
    edges = _golden_edges(name)
    eng = _engine(edges, v_num)
    dev = eng.graph.csr()
    ref = oracle.Csr(edges, v_num, undirected=True)
    np.testing.assert_array_equal(dev["offsets"], ref.offsets)
    np.testing.assert_array_equal(dev["nbr"], ref.nbr)
    np.testing.assert_array_equal(dev["out_deg"], ref.out_deg)
    np.testing.assert_array_equal(dev["in_deg"], ref.in_deg)
    np.testing.assert_array_equal(dev["thresholds"], ref.thresholds())


def test_c1_thresholds_bit_exact(distger_lib, oracle, c1_edges):
    eng = _engine(c1_edges, 10_000)
    ref = oracle.Csr(c1_edges, 10_000, undirected=True)
    thr = eng.graph.csr()["thresholds"]
    np.testing.assert_array_equal(thr, ref.thresholds())


@pytest.mark.parametrize("name,v_num,min_r", [("tiny200", 200, 5), ("special60", 60, 3)])
def test_all_rounds_bit_exact(distger_lib, oracle, name, v_num, min_r, tmp_path):
    edges = _golden_edges(name)
    seed = 0x5EED0001
    eng = _engine(edges, v_num, seed=seed, min_r=min_r)
    ref = oracle.Csr(edges, v_num, undirected=True)
    want, st = oracle.walk_rounds(ref, v_num, 20, min_r, 30, seed=seed)
    freq = np.zeros(v_num, np.int64)
    prev_h = None
    steps = draws = traces = 0
    for r in range(1, 31):
        paths = eng.run_round(v_num, r)
        offs, verts = paths.to_numpy()
        np.testing.assert_array_equal(offs, want[r - 1][0], err_msg=f"round {r}")
        np.testing.assert_array_equal(verts, want[r - 1][1], err_msg=f"round {r}")
        freq += np.bincount(verts, minlength=v_num)
        h = oracle.relative_entropy(ref.out_deg, freq.astype(np.uint32))
        assert paths.info.relative_entropy == pytest.approx(h, rel=1e-9, abs=1e-15)
        if prev_h is not None:
            assert paths.info.delta_h == pytest.approx(h - prev_h, rel=1e-6, abs=1e-12)
        prev_h = h
        steps += paths.info.steps
        draws += paths.info.draws
        traces += paths.info.traces
        if r in (1, 30):
            out = str(tmp_path / f"w-0-{r}.txt")
            paths.write_text(out)
            assert open(out, "rb").read() == oracle.walk_text(offs, verts)
        paths.close()
    assert (steps, draws, traces) == (st.steps, st.draws, st.traces)
    np.testing.assert_array_equal(eng.graph.visits(), freq)


def test_c1_round_bit_exact(distger_lib, oracle, c1_edges):
    """C1 small config (10k vertices, 100k edges): rounds 1-3 bit-exact."""
    eng = _engine(c1_edges, 10_000, seed=42)
    ref = oracle.Csr(c1_edges, 10_000, undirected=True)
    want, st = oracle.walk_rounds(ref, 10_000, 20, 5, 3, seed=42)
    for r in range(1, 4):
        paths = eng.run_round(10_000, r)
        offs, verts = paths.to_numpy()
        np.testing.assert_array_equal(offs, want[r - 1][0])
        np.testing.assert_array_equal(verts, want[r - 1][1])


def test_directed_graph_with_sinks(distger_lib, oracle):
    """Without --make-undirected some vertices have out-degree 0: walks stop there."""
    from distger import graphgen
    edges = graphgen.chung_lu(500, 1500, 2.2, seed=5)
    eng = _engine(edges, 500, undirected=False, seed=7)
    ref = oracle.Csr(edges, 500, undirected=False)
    assert (ref.out_deg == 0).any()
    want, _ = oracle.walk_rounds(ref, 500, 20, 5, 2, seed=7)
    for r in (1, 2):
        offs, verts = eng.run_round(500, r).to_numpy()
        np.testing.assert_array_equal(offs, want[r - 1][0])
        np.testing.assert_array_equal(verts, want[r - 1][1])


def test_edgeless_graph(distger_lib):
    edges = np.zeros(0, dtype=[("src", "<u4"), ("dst", "<u4"), ("data", "<f4")])
    eng = _engine(edges, 5, seed=1)
    offs, verts = eng.run_round(5, 1).to_numpy()
    np.testing.assert_array_equal(np.diff(offs.astype(np.int64)), np.ones(25))
    np.testing.assert_array_equal(verts, np.arange(25) % 5)


def test_overflow_is_an_error_and_leaves_state_unchanged(distger_lib, oracle):
    from distger import DistgerError
    edges = _golden_edges("tiny200")
    eng = _engine(edges, 200, seed=9, max_len=8)
    with pytest.raises(DistgerError) as e:
        eng.run_round(200, 1)
    assert e.value.code == -5
    assert int(eng.graph.visits().sum()) == 0
    eng.max_len = 64
    offs, verts = eng.run_round(200, 1).to_numpy()
    ref = oracle.Csr(edges, 200, undirected=True)
    want, _ = oracle.walk_rounds(ref, 200, 20, 5, 1, seed=9)
    np.testing.assert_array_equal(verts, want[0][1])


def test_youtube_shaped_round_sampled_exact(distger_lib, oracle):
    """Full C2 size (1,138,499 vertices, ~3M edges): round 1 with 10 walkers per
    vertex; 3000 sampled walker ids bit-exact against the checker, plus
    size-independent properties over every walk."""
    from distger import graphgen
    cfg = graphgen.CONFIGS["c2_youtube"]
    edges = graphgen.chung_lu(**cfg)
    v_num = cfg["n"]
    eng = _engine(edges, v_num, seed=2024, min_r=10)
    paths = eng.run_round(v_num, 1)
    info = paths.info
    offs, verts = paths.to_numpy()
    n = v_num * 10
    assert info.n_walks == n and offs.size == n + 1
    lens = np.diff(offs.astype(np.int64))
    starts = verts[offs[:-1].astype(np.int64)]
    np.testing.assert_array_equal(starts, np.arange(n, dtype=np.int64) % v_num)
    assert info.steps == verts.size - n
    # Every walk ends by the entropy test (>= min_len + 2 footprints) or a guard.
    assert lens.min() >= 1 and lens.max() <= 64
    ref = oracle.Csr(edges, v_num, undirected=True)
    ids = np.random.default_rng(0).choice(n, size=3000, replace=False).astype(np.uint32)
    w_offs, w_verts = oracle.walk_ids(ref, ids, 1, 20, seed=2024)
    for i, w in enumerate(ids):
        np.testing.assert_array_equal(verts[offs[w]:offs[w + 1]], w_verts[w_offs[i]:w_offs[i + 1]])
    # Visit frequencies equal the histogram of the footprints.
    np.testing.assert_array_equal(eng.graph.visits(), np.bincount(verts, minlength=v_num))
    # Replay: the same round again gives identical walks.
    offs2, verts2 = eng.run_round(v_num, 1).to_numpy()
    np.testing.assert_array_equal(verts2, verts)
