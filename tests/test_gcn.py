"""Common-neighbour counts: the CPU restatement against the reference's own gcn
tool (golden fixtures written by tests/golden/make_gcn_golden.py from the tool
compiled unmodified, and the live tool when it is built)."""
import os
import subprocess

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = [("multi60", 60), ("hubs300", 300), ("tiny200", 200)]


def _read(name):
    e = np.loadtxt(os.path.join(GOLDEN, f"gcn_{name}.in.txt"), dtype=np.int64).reshape(-1, 2)
    out = np.loadtxt(os.path.join(GOLDEN, f"gcn_{name}.out.txt"), dtype=np.int64).reshape(-1, 3)
    return e, out


@pytest.mark.parametrize("name,v", CASES)
def test_restatement_matches_reference_fixtures(oracle, name, v):
    e, out = _read(name)
    assert np.array_equal(out[:, :2], e)
    got = oracle.common_neighbours(e[:, 0], e[:, 1], v, undirected=True)
    assert np.array_equal(got, out[:, 2])


def test_restatement_matches_live_reference(oracle, tmp_path):
    tool = os.path.join(os.path.dirname(oracle.HERE), "oracle", "_ref", "gcn_ref")
    if not os.path.exists(tool):
        pytest.skip("reference gcn tool not built (make -C oracle ref)")
    rng = np.random.default_rng(5)
    for trial in range(6):
        v = int(rng.integers(5, 120))
        e = rng.integers(0, v, size=(int(rng.integers(1, 800)), 2))
        inp, outp = tmp_path / f"g{trial}.txt", tmp_path / f"o{trial}.txt"
        inp.write_text("".join(f"{a} {b}\n" for a, b in e.tolist()))
        subprocess.run([tool, "-i", str(inp), "-o", str(outp), "-v", str(v), "-t", "1", "-s", "unweighted",
                        "--make-undirected"], check=True, capture_output=True)
        want = np.loadtxt(outp, dtype=np.int64).reshape(-1, 3)[:, 2]
        assert np.array_equal(oracle.common_neighbours(e[:, 0], e[:, 1], v), want), trial
