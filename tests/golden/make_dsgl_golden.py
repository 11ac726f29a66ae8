"""Golden fixtures of the reference's own dsgl trainer.

Runs include/dsgl.hpp's dsgl() unmodified (oracle/_ref/ref_dsgl, built by
`make -C oracle ref REF=<reference>`: one-rank MPI and naive-GEMM stand-ins,
-threads 2 = one compute thread, a model-sync period longer than the run) on the
seeded corpora of tests/dsgl_cases.py and writes dsgl_ref.json: per case the
sha256 of the final Wih and Woh rows (vocabulary order), the vocabulary order's
digest and the final learning rate.
Usage: python tests/golden/make_dsgl_golden.py
"""
import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

import dgoracle  # noqa: E402
import dsgl_cases  # noqa: E402


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    out = {}
    for name in dsgl_cases.CASES:
        c = dsgl_cases.make_case(name)
        with tempfile.TemporaryDirectory() as tmp:
            ids, wih, woh, alpha = dgoracle.run_ref_dsgl(tmp, c["counts"], c["corpus"], c["size"], c["window"],
                                                         c["negative"], c["sample"], c["alpha"], c["iterations"],
                                                         sync_period=20.0)
        out[name] = {"ids": digest(ids), "wih": digest(wih), "woh": digest(woh), "alpha": float(alpha)}
        print(name, out[name]["wih"][:16], out[name]["woh"][:16], alpha)
    with open(os.path.join(HERE, "dsgl_ref.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
