"""Writes the common-neighbour golden fixtures from the reference's own gcn tool.

Run from the repository root after `make -C oracle ref` (oracle/_ref/gcn_ref is
src/tools/gcn.cpp compiled unmodified with the one-rank MPI stand-in):

    python tests/golden/make_gcn_golden.py

Each case writes gcn_<name>.in.txt (the tool's input, "src dst" per line) and
gcn_<name>.out.txt (its output with -t 1 --make-undirected).
"""
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TOOL = os.path.join(HERE, "..", "..", "oracle", "_ref", "gcn_ref")


def cases():
    rng = np.random.default_rng(20)
    # a multigraph with self-loops and repeated pairs in both orientations
    yield "multi60", 60, rng.integers(0, 60, size=(400, 2))
    # a power-law graph with hubs (pairs drawn proportional to i^-1.2)
    w = 1.0 / np.arange(1, 301) ** 1.2
    p = w / w.sum()
    yield "hubs300", 300, np.stack([rng.choice(300, 3000, p=p), rng.choice(300, 3000, p=p)], axis=1)
    # the walk fixtures' graph
    rec = np.fromfile(os.path.join(HERE, "tiny200.bin"), dtype=np.dtype([("s", "<u4"), ("d", "<u4"), ("w", "<f4")]))
    yield "tiny200", 200, np.stack([rec["s"], rec["d"]], axis=1)


def main():
    for name, v, e in cases():
        inp = os.path.join(HERE, f"gcn_{name}.in.txt")
        out = os.path.join(HERE, f"gcn_{name}.out.txt")
        with open(inp, "w") as f:
            for a, b in e.tolist():
                f.write(f"{a} {b}\n")
        subprocess.run([TOOL, "-i", inp, "-o", out, "-v", str(v), "-t", "1", "-s", "unweighted",
                        "--make-undirected"], check=True, capture_output=True)
        print(name, len(e))


if __name__ == "__main__":
    main()
