"""The C++ host program (bin/huge_walk) and the one-call embedding job (distger.embed).

huge_walk's walk files must equal the CPU checker's walk text byte for byte, and
in deterministic mode its embedding must equal the kernel-order FP32 checker fed
the same walks with the same per-round learning rates.
"""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "gdistger-re_b200", "bin", "huge_walk")
GOLDEN = os.path.join(ROOT, "tests", "golden")
pytestmark = pytest.mark.gpu


def _run(args):
    assert os.path.exists(EXE), "huge_walk not built (make -C gdistger-re_b200/csrc)"
    r = subprocess.run([EXE] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


def test_huge_walk_files_and_embedding_bit_exact(distger_lib, oracle, tmp_path):
    from distger import graphgen, lp
    edges_path = os.path.join(GOLDEN, "tiny200.bin")
    edges = graphgen.read_edges(edges_path)
    seed, rounds = 31, 3
    prefix = str(tmp_path / "walks")
    emb_path = str(tmp_path / "emb.txt")
    out = _run(["-g", edges_path, "-v", "200", "-w", "200", "--min_L", "20", "--min_R", "5", "--make-undirected",
                "-o", prefix, "-size", "64", "-window", "5", "-negative", "5", "-sample", "1e-3", "-alpha", "0.025",
                "-iter", "1", "-min-count", "0", "-emb_output", emb_path, "-mode", "plain", "-deterministic", "1",
                "-seed", str(seed), "-rounds", str(rounds), "-table-size", "100000", "-train-from", "1"])
    alphas = [float(a) for a in re.findall(r"alpha (\S+) walk", out)]
    assert len(alphas) == rounds and alphas[0] == pytest.approx(0.025)
    csr = oracle.Csr(edges, 200, undirected=True)
    want, _ = oracle.walk_rounds(csr, 200, 20, 5, rounds, seed=seed)
    for r in range(1, rounds + 1):
        assert open(f"{prefix}-0-{r}.txt", "rb").read() == oracle.walk_text(*want[r - 1])
    counts = (csr.out_deg + csr.in_deg).astype(np.uint32)
    o = oracle.Sgns(counts, size=64, window=5, negative=5, sample=1e-3, alpha=0.025, min_count=0, seed=seed,
                    table_size=100_000)
    for r in range(rounds):
        o.train(*want[r], alpha=np.float32(alphas[r]))
    got = lp.read_embedding_text(emb_path, 200)
    with open(emb_path) as f:
        assert f.readline().split() == ["200", "64"]
    # The text holds "%lf" (6 decimals) of the FP32 rows.
    ids = np.flatnonzero(counts > 0)
    np.testing.assert_allclose(got[ids], _by_vertex(o, 200)[ids], atol=6e-7, rtol=0)


def _by_vertex(o, v_num):
    emb = np.zeros((v_num, o.syn0_f32.shape[1]), np.float32)
    emb[o.vocab_ids] = o.syn0_f32
    return emb


def test_huge_walk_reference_defaults(distger_lib, oracle, tmp_path):
    """No -mode: -cbow 1 (word2vec.cu:59) trains cbow_kernel's rule; rounds 1-2 are
    walked but not trained and the schedule starts at 0.025 whatever -alpha says
    (word2vec.cu:1279-1290); run.sh's dsgl flags are accepted."""
    from distger import graphgen, lp
    edges_path = os.path.join(GOLDEN, "tiny200.bin")
    edges = graphgen.read_edges(edges_path)
    emb_path = str(tmp_path / "emb.txt")
    seed, rounds = 5, 4
    out = _run(["-g", edges_path, "-v", "200", "-w", "200", "--min_L", "20", "--min_R", "5", "--make-undirected",
                "-size", "64", "-iter", "1", "-threads", "10", "-window", "5", "-negative", "5", "-batch-size", "21",
                "-min-count", "0", "-sample", "1e-3", "-alpha", "0.01", "-debug", "2", "-sync-size", "1024",
                "-emb_output", emb_path, "-deterministic", "1", "-seed", str(seed), "-rounds", str(rounds),
                "-table-size", "100000"])
    assert "mode cbow" in out
    assert out.count("(not trained)") == 2
    alphas = [float(a) for a in re.findall(r"alpha (\S+) walk", out)]
    assert alphas == [pytest.approx(0.025), pytest.approx(0.025 * np.exp(np.float32(-0.1)))]
    csr = oracle.Csr(edges, 200, undirected=True)
    want, _ = oracle.walk_rounds(csr, 200, 20, 5, rounds, seed=seed)
    counts = (csr.out_deg + csr.in_deg).astype(np.uint32)
    o = oracle.Sgns(counts, size=64, window=5, negative=5, sample=1e-3, alpha=0.05, min_count=0, seed=seed,
                    table_size=100_000)
    for r in (2, 3):
        o.train(*want[r], alpha=np.float32(alphas[r - 2]), rule="cbow")
    got = lp.read_embedding_text(emb_path, 200)
    ids = np.flatnonzero(counts > 0)
    np.testing.assert_allclose(got[ids], _by_vertex(o, 200)[ids], atol=6e-7, rtol=0)


def test_huge_walk_run_sh_flags(distger_lib, tmp_path):
    """The reference's run.sh learning flags (build/run.sh:60-71) verbatim, on the
    tiny graph: -size 100 (stored padded to 128 columns), -iter 3, -threads 10,
    -sync-size 1024; CBOW by default.  The embedding has 100 columns."""
    from distger import lp
    edges_path = os.path.join(GOLDEN, "tiny200.bin")
    emb_path = str(tmp_path / "emb.txt")
    out = _run(["-g", edges_path, "-v", "200", "-w", "200", "--min_L", "20", "--min_R", "1", "-o",
                str(tmp_path / "walks"), "--make-undirected", "-emb_output", emb_path, "-size", "100", "-iter", "3",
                "-threads", "10", "-window", "10", "-negative", "5", "-batch-size", "21", "-min-count", "0",
                "-sample", "1e-3", "-alpha", "0.01", "-debug", "2", "-sync-size", "1024", "-rounds", "4",
                "-table-size", "100000"])
    assert "mode cbow" in out
    with open(emb_path) as f:
        assert f.readline().split() == ["200", "100"]
        row = f.readline().split()
    assert len(row) == 101
    emb = lp.read_embedding_text(emb_path, 200)
    assert emb.shape == (200, 100) and np.isfinite(emb).all() and np.abs(emb).max() > 0


def test_huge_walk_rejects_bad_flags():
    r = subprocess.run([EXE, "-g", "x.bin", "-v", "10", "-w", "10", "-binary", "1"], capture_output=True, text=True)
    assert r.returncode == 2 and "not supported" in r.stderr
    r = subprocess.run([EXE, "-g", "x.bin", "-v", "10"], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def test_embed_job_runs_all_rounds(distger_lib):
    import distger
    from distger import graphgen
    from distger.embed import embed
    edges = graphgen.chung_lu(2000, 20_000, 2.2, seed=4)
    g = distger.Graph(2000, edges=edges, make_undirected=True)
    res = embed(g, mode="minibatch", size=64, window=5, rounds=30)
    assert len(res["rounds"]) == 30
    assert res["rounds"][0]["walks"] == 2000 * 5 and res["rounds"][1]["walks"] == 2000
    assert res["words"] > 0 and res["embedding"].shape == (2000, 64)
    assert np.isfinite(res["embedding"]).all() and np.abs(res["embedding"]).max() > 0
    g.close()
