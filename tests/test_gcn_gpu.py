"""Device common-neighbour counts against the reference's gcn tool (golden
fixtures from the tool itself) and against the CPU restatement; the C++ host
program's output file must equal the tool's byte for byte."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,v", [("multi60", 60), ("hubs300", 300), ("tiny200", 200)])
def test_device_counts_match_reference_tool(distger_lib, name, v, tmp_path):
    from distger.synth import common_neighbours
    e = np.loadtxt(os.path.join(GOLDEN, f"gcn_{name}.in.txt"), dtype=np.int64).reshape(-1, 2)
    want = np.loadtxt(os.path.join(GOLDEN, f"gcn_{name}.out.txt"), dtype=np.int64).reshape(-1, 3)[:, 2]
    assert np.array_equal(common_neighbours(e[:, 0], e[:, 1], v), want)
    out, binf = tmp_path / "out.txt", tmp_path / "out.bin"
    r = subprocess.run([os.path.join(ROOT, "gdistger-re_b200", "bin", "gcn"), "-i",
                        os.path.join(GOLDEN, f"gcn_{name}.in.txt"), "-o", str(out), "-v", str(v), "-t", "1", "-s",
                        "unweighted", "--make-undirected", "-b", str(binf)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert out.read_bytes() == open(os.path.join(GOLDEN, f"gcn_{name}.out.txt"), "rb").read()
    rec = np.fromfile(binf, dtype=np.dtype([("s", "<u4"), ("d", "<u4"), ("w", "<f4")]))
    assert np.array_equal(rec["w"], want.astype(np.float32)) and np.array_equal(rec["s"], e[:, 0])


@pytest.mark.parametrize("undirected", [True, False])
def test_device_counts_match_restatement_on_power_law_graph(distger_lib, oracle, undirected):
    from distger import graphgen
    from distger.synth import common_neighbours
    e = graphgen.chung_lu(10_000, 100_000, 2.2, seed=3)
    src, dst = e["src"].astype(np.int64), e["dst"].astype(np.int64)
    # repeat a few pairs, in both orientations, and add self-loops
    src = np.concatenate([src, dst[:500], src[:300], np.arange(50)])
    dst = np.concatenate([dst, src[:500], dst[:300], np.arange(50)])
    got = common_neighbours(src, dst, 10_000, undirected=undirected)
    assert np.array_equal(got, oracle.common_neighbours(src, dst, 10_000, undirected=undirected))
