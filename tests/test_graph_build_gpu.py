"""The device CSR build of loaded records (dg_graph_create / _from_edges):
bit-exact against the CPU checker's CSR in record order (the reference's
bucketing) on adversarial multigraphs -- self-loops, repeated records, sinks,
directed and undirected, a vertex range wider than the ids used -- and the
reference's input errors reported as DG_ERR_ARG with the first bad record."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = [("src", "<u4"), ("dst", "<u4"), ("data", "<f4")]


def _records(n, v, seed, self_loops=0.1, repeats=0.1):
    rng = np.random.default_rng(seed)
    e = np.zeros(n, dtype=DT)
    e["src"] = rng.integers(0, v, n)
    e["dst"] = rng.integers(0, v, n)
    loop = rng.random(n) < self_loops
    e["dst"][loop] = e["src"][loop]
    rep = rng.random(n) < repeats
    idx = np.flatnonzero(rep)
    if idx.size:
        e[idx] = e[rng.integers(0, n, idx.size)]
    e["data"] = rng.integers(1, 5, n).astype(np.float32) * rng.choice([1.0, 0.5, 0.25], n).astype(np.float32)
    return e


@pytest.mark.parametrize("undirected", [True, False])
@pytest.mark.parametrize("n,v,seed", [(5_000, 300, 1), (200_000, 70_000, 2), (1, 1, 3)])
def test_csr_record_order_bit_exact(distger_lib, oracle, undirected, n, v, seed):
    from distger import Graph
    e = _records(n, v, seed)
    g = Graph(v + 7, edges=e, make_undirected=undirected)   # ids above the largest one used have no edges
    dev = g.csr()
    ref = oracle.Csr(e, v + 7, undirected=undirected)
    np.testing.assert_array_equal(dev["offsets"], ref.offsets)
    np.testing.assert_array_equal(dev["nbr"], ref.nbr)
    np.testing.assert_array_equal(dev["out_deg"], ref.out_deg)
    np.testing.assert_array_equal(dev["in_deg"], ref.in_deg)
    np.testing.assert_array_equal(dev["thresholds"], ref.thresholds())
    g.close()


def test_file_load_matches_records(distger_lib, oracle, tmp_path):
    from distger import Graph, graphgen
    e = _records(50_000, 4_000, 4)
    path = tmp_path / "g.bin"
    graphgen.write_edges(str(path), e)
    a, b = Graph(4_000, graph_path=str(path), make_undirected=True), Graph(4_000, edges=e, make_undirected=True)
    ca, cb = a.csr(), b.csr()
    for k in ca:
        np.testing.assert_array_equal(ca[k], cb[k])
    a.close()
    b.close()


@pytest.mark.parametrize("bad,what", [((2, 10, 0.5), "vertex id"), ((1, 2, float("nan")), "data"),
                                      ((1, 2, 3e9), "data"), ((1, 2, float("inf")), "data")])
def test_bad_records_are_errors(distger_lib, bad, what):
    from distger import DistgerError, Graph
    e = _records(1000, 10, 5)
    e[[400, 700]] = bad
    with pytest.raises(DistgerError) as err:
        Graph(10, edges=e, make_undirected=True)
    assert err.value.code == -1
    assert "edge 400" in str(err.value) and what in str(err.value)
