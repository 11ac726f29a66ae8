"""The CPU checker for the walk, pinned against the reference's own engine.

The golden fixtures under tests/golden/ were written by the UNMODIFIED reference
walk engine (tests/golden/make_golden.py); when the reference tree is present the
comparison is also repeated live against a freshly built oracle/_ref/ref_walk.
"""
import os
import subprocess

import numpy as np
import pytest

import dgoracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _edges(name):
    from distger import graphgen
    return graphgen.read_edges(os.path.join(GOLDEN, f"{name}.bin"))


def test_philox_known_answers(oracle):
    # Random123 known-answer vectors for Philox4x32-10.
    assert oracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


@pytest.mark.parametrize("name", ["tiny200", "special60"])
def test_oracle_reproduces_reference_walk_files(oracle, name):
    rounds, abs_dh, meta = oracle.load_golden(os.path.join(GOLDEN, f"{name}_ref_walks.npz"))
    v_num, walkers, min_len, min_r, seed = (int(x) for x in meta)
    csr = oracle.Csr(_edges(name), v_num, undirected=True)
    mine, stats = oracle.walk_rounds(csr, walkers, min_len, min_r, 30, stream_seed=seed)
    assert len(mine) == len(rounds) == 30
    freq = np.zeros(v_num, np.int64)
    prev = None
    for r, ((mo, mv), (go, gv)) in enumerate(zip(mine, rounds), start=1):
        np.testing.assert_array_equal(mo, go, err_msg=f"round {r} offsets")
        np.testing.assert_array_equal(mv, gv, err_msg=f"round {r} vertices")
        # Relative entropy of cumulative visits vs degree share, as the engine printed it.
        freq += np.bincount(mv, minlength=v_num)
        h = oracle.relative_entropy(csr.out_deg, freq.astype(np.uint32))
        dh = h if prev is None else h - prev
        prev = h
        assert abs(abs(dh) - abs_dh[r - 1]) <= 5e-6 * abs(abs_dh[r - 1]) + 1e-12
    assert stats.pow_sq_mismatch == 0


def test_special_graph_corner_cases(oracle):
    rounds, _, meta = oracle.load_golden(os.path.join(GOLDEN, "special60_ref_walks.npz"))
    offs, verts = rounds[0]
    v_num = int(meta[0])
    starts = verts[offs[:-1].astype(np.int64)]
    lens = np.diff(offs.astype(np.int64))
    # Vertex 7's adjacency is [7, 7]: walks from it stop before any step (walk.hpp:900-902).
    assert np.all(lens[starts == 7] == 1)
    # Everyone else walks at least min_len + 2 footprints.
    assert np.all(lens[starts != 7] >= 22)
    assert set(np.unique(starts)) == set(range(v_num))


def test_oracle_philox_walk_properties(oracle):
    csr = oracle.Csr(_edges("tiny200"), 200, undirected=True)
    rounds, st = oracle.walk_rounds(csr, 200, 20, 5, 3, seed=1234)
    assert len(rounds) == 3
    for r, (offs, verts) in enumerate(rounds, start=1):
        n = 200 * 5 if r == 1 else 200
        assert offs.size == n + 1
        starts = verts[offs[:-1].astype(np.int64)]
        np.testing.assert_array_equal(starts, np.arange(n) % 200)
        # Every step moves along an edge of the CSR.
        for w in range(0, n, 37):
            seg = verts[offs[w]:offs[w + 1]]
            for a, b in zip(seg[:-1], seg[1:]):
                row = csr.nbr[csr.offsets[a]:csr.offsets[a + 1]]
                assert b in row
    # Seeded replay is deterministic and seed-sensitive.
    again, _ = oracle.walk_rounds(csr, 200, 20, 5, 1, seed=1234)
    np.testing.assert_array_equal(again[0][1], rounds[0][1])
    other, _ = oracle.walk_rounds(csr, 200, 20, 5, 1, seed=1235)
    assert not np.array_equal(other[0][1], rounds[0][1])


def test_thresholds_match_the_acceptance_test(oracle):
    """k >= threshold  <=>  tanh(p_accept) <= k / RAND_MAX  (walk.hpp:928-942)."""
    csr = oracle.Csr(_edges("special60"), 60, undirected=True)
    thr = csr.thresholds()
    rng = np.random.default_rng(0)
    for e in rng.choice(csr.m, size=200, replace=False):
        v = int(np.searchsorted(csr.offsets, e, side="right") - 1)
        sd, dd, cn = int(csr.out_deg[v]), int(csr.out_deg[csr.nbr[e]]), int(csr.data[e])
        pa = (1 / float(sd - cn)) * float(max(sd, dd)) / min(sd, dd) if sd != cn else float("inf")
        t = np.tanh(pa)
        k = int(thr[e])
        if k <= 2147483647:
            assert t <= k / 2147483647.0
        if 0 < k <= 2147483647:
            assert not (t <= (k - 1) / 2147483647.0)


@pytest.mark.skipif(not (os.path.exists(dgoracle.REF_WALK) and os.path.exists(dgoracle.REF_WALK_FMA)),
                    reason="reference engine not built (make -C oracle ref REF=<reference tree>)")
def test_oracle_matches_live_reference(oracle, tmp_path):
    """Runs the reference engine (built from its sources into oracle/_ref) and
    compares on a fresh graph."""
    from distger import graphgen
    assert oracle.build_ref()
    edges = graphgen.chung_lu(1500, 9000, 2.1, seed=3)
    path = str(tmp_path / "g.bin")
    graphgen.write_edges(path, edges)
    for exe in (oracle.REF_WALK, oracle.REF_WALK_FMA):
        prefix = str(tmp_path / os.path.basename(exe))
        subprocess.run([exe, "-g", path, "-v", "1500", "-w", "1500", "--min_L", "20", "--min_R", "2",
                        "-o", prefix, "--make-undirected", "-t", "1", "--seed", "99"],
                       check=True, capture_output=True)
        csr = oracle.Csr(edges, 1500, undirected=True)
        mine, _ = oracle.walk_rounds(csr, 1500, 20, 2, 30, stream_seed=99)
        for r in (1, 2, 17, 30):
            assert oracle.walk_text(*mine[r - 1]) == open(f"{prefix}-0-{r}.txt", "rb").read()
