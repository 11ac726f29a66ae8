"""Golden fixtures of the reference's own word2vec.cu kernels.

Runs skip_gram_kernel, cbow_kernel and __sgNegReuse, compiled unmodified for
sm_100a into oracle/_ref/libref_w2v.so (`make -C oracle ref REF=<reference>`),
on the seeded cases of tests/w2v_cases.py, one sentence per launch, and writes
  w2v_ref.json        sha256 of the final rows of every case
  w2v_reuse200.npz    the final rows of the __sgNegReuse case (compared with a
                      tolerance: that kernel sums a pair's updates with shared-
                      memory atomics in warp arrival order)
Needs a GPU.  Usage: python tests/golden/make_w2v_golden.py [out_dir]
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

import w2v_cases as W  # noqa: E402


def main(out_dir: str) -> None:
    os.makedirs(out_dir, exist_ok=True)
    ref = {}
    et = W.exp_table()
    for name in W.CASES:
        c = W.make_case(name)
        table = W.unigram_table(c["counts"])
        s0, s1 = W.run_reference_kernels(c, table, et)
        ref[name] = {"syn0": W.digest(s0), "syn1": W.digest(s1)}
        if c["kind"] == 2:
            np.savez_compressed(os.path.join(out_dir, f"w2v_{name}.npz"), syn0=s0, syn1=s1)
        print(name, ref[name]["syn0"][:16], ref[name]["syn1"][:16])
    with open(os.path.join(out_dir, "w2v_ref.json"), "w") as f:
        json.dump(ref, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
