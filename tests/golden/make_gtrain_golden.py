"""Golden digests of the reference's gtrain split (src/tools/gtrain.cpp), run
unmodified (oracle/_ref/gtrain_ref, built by `make -C oracle ref`) with
oracle/_ref/fixed_time.so preloaded, so that its srand(time(0)) takes the seed
named here.  Writes tests/golden/gtrain_ref.json: per case the graph's
generator arguments, the seed and fraction, and the sha256 of the tool's three
output files (train edges, test pairs, test labels).  The graph of a case is
regenerated by tests/test_lp.py with `case_edges`.
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")

# name: (vertices, draws, graph seed, split seed, fraction)
CASES = {
    "small": (300, 2000, 1, 12345, 0.1),
    "mid": (3000, 30000, 2, 777, 0.1),
    "dense_holdout": (500, 6000, 3, 4242, 0.3),
}


def case_edges(name: str) -> np.ndarray:
    """Random directed pairs without self-loops and integer data 1..8, in file order."""
    sys.path.insert(0, os.path.join(ROOT, "gdistger-re_b200"))
    from distger import graphgen
    n, draws, gseed, _, _ = CASES[name]
    rng = np.random.default_rng(gseed)
    src = rng.integers(0, n, draws)
    dst = rng.integers(0, n, draws)
    data = rng.integers(1, 9, draws)
    keep = src != dst
    e = np.zeros(int(keep.sum()), dtype=graphgen.EDGE_DTYPE)
    e["src"], e["dst"], e["data"] = src[keep], dst[keep], data[keep]
    return e


def write_edges(e: np.ndarray, path: str) -> None:
    with open(path, "w") as f:
        for a, b, c in zip(e["src"].tolist(), e["dst"].tolist(), e["data"].astype(np.int64).tolist()):
            f.write(f"{a}\t{b}\t{c}\n")


def run_ref(name: str, workdir: str):
    n, _, _, seed, frac = CASES[name]
    g = os.path.join(workdir, "g.txt")
    write_edges(case_edges(name), g)
    out = [os.path.join(workdir, x) for x in ("lp.txt", "te.txt", "tl.txt")]
    env = dict(os.environ, DG_FIXED_TIME=str(seed), LD_PRELOAD=os.path.join(REF, "fixed_time.so"))
    subprocess.run([os.path.join(REF, "gtrain_ref"), "-i", g, "-o", out[0], "-e", out[1], "-l", out[2], "-s",
                    str(frac), "-v", str(n), "-t", "1"], env=env, check=True, capture_output=True)
    return [open(p, "rb").read() for p in out]


def main():
    res = {}
    for name in CASES:
        with tempfile.TemporaryDirectory() as d:
            files = run_ref(name, d)
        res[name] = {"case": list(CASES[name]), "sha256": [hashlib.sha256(b).hexdigest() for b in files],
                     "lines": [b.count(b"\n") for b in files]}
    with open(os.path.join(HERE, "gtrain_ref.json"), "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
