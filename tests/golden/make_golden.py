"""Regenerates the walk golden fixtures from the reference's own walk engine.

Run where the reference tree is (its path in DG_REFERENCE_DIR):
  DG_REFERENCE_DIR=<reference tree> python tests/golden/make_golden.py

For each small graph it writes <name>.bin (packed 12-byte edge records) and
<name>_ref_walks.npz: the 30 per-round walk files produced by the UNMODIFIED
reference engine (oracle/_ref/ref_walk, built by `make -C oracle ref`; one worker
thread, mt19937 seed pinned to 5489, glibc rand() from its default state), stored
as per-round (offsets, vertices) arrays, plus the |delta H| values the engine
printed after each round (walk.hpp:729, six significant digits).
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gdistger-re_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from distger import graphgen  # noqa: E402
import dgoracle  # noqa: E402

PINNED_SEED = 5489


def special_graph() -> tuple[np.ndarray, int]:
    """60 vertices: power-law core plus the transition's corner cases.

    - vertex 3 carries a self-loop (step-0 resampling, walk.hpp:904-906);
    - vertex 7's only record is a self-loop, so after doubling its adjacency is
      [7, 7] and every walk from it ends at once (deg == 2 guard, walk.hpp:900-902);
    - some records carry data exactly 1.0, so (int)data = 1 (walk.hpp:920).
    """
    n = 60
    e = graphgen.chung_lu(n, 200, 2.2, seed=7)
    e = e[(e["src"] != 7) & (e["dst"] != 7)]
    extra = np.zeros(3, dtype=graphgen.EDGE_DTYPE)
    extra[0] = (7, 7, 0.5)
    extra[1] = (3, 3, 0.25)
    extra[2] = (3, 11, 1.0)
    e = np.concatenate([extra[:1], e, extra[1:]])
    e["data"][::9] = np.float32(1.0)
    return e, n


def graphs():
    yield "tiny200", graphgen.chung_lu(200, 1000, 2.2, seed=0), 200, 5
    e, n = special_graph()
    yield "special60", e, n, 3


def main() -> None:
    if not dgoracle.build_ref():
        raise SystemExit("reference tree not found; set DG_REFERENCE_DIR")
    for name, edges, v_num, min_r in graphs():
        bin_path = os.path.join(HERE, f"{name}.bin")
        graphgen.write_edges(bin_path, edges)
        with tempfile.TemporaryDirectory() as tmp:
            prefix = os.path.join(tmp, "w")
            out = subprocess.run([dgoracle.REF_WALK, "-g", bin_path, "-v", str(v_num), "-w", str(v_num),
                                  "--min_L", "20", "--min_R", str(min_r), "-o", prefix, "--make-undirected",
                                  "-t", "1", "--seed", str(PINNED_SEED)],
                                 check=True, capture_output=True, text=True).stdout
            arrays = {}
            for r in range(1, 31):
                lines = open(f"{prefix}-0-{r}.txt").read().split("\n")[:-1]
                walks = [[int(x) for x in ln.split()] for ln in lines]
                lens = np.array([len(w) for w in walks], dtype=np.uint64)
                arrays[f"offsets_{r}"] = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
                arrays[f"verts_{r}"] = np.array([x for w in walks for x in w], dtype=np.uint32)
        dh = [float(x) for x in re.findall(r"abs\(delta_H\) = ([0-9.eE+-]+)", out)]
        arrays["abs_delta_h"] = np.array(dh, dtype=np.float64)
        arrays["meta"] = np.array([v_num, v_num, 20, min_r, PINNED_SEED], dtype=np.int64)
        np.savez_compressed(os.path.join(HERE, f"{name}_ref_walks.npz"), **arrays)
        print(name, "rounds", len(dh), "walks/round1", arrays["offsets_1"].size - 1)


if __name__ == "__main__":
    main()
