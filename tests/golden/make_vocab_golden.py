"""Golden digests of word2vec.cu's own vocabulary from degrees (ReadVocabFromDegree
+ SortVocab, run from oracle/_ref/libref_w2v.so, the reference compiled
unmodified): per case the vocabulary size, train_words and the sha256 of the
vertex ids in vocabulary order.  Writes tests/golden/w2v_vocab_ref.json; the
graphs are regenerated by tests/test_oracle_vocab.py with `case_counts`."""
import ctypes as C
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

# name: (vertices, edges drawn (0: the tiny200 golden graph), Chung-Lu exponent, seed, min_count)
CASES = {
    "tiny200_mc0": (200, 0, 0.0, 0, 0),
    "tiny200_mc5": (200, 0, 0.0, 0, 5),
    "cl10k_mc0": (10_000, 100_000, 2.2, 0, 0),
    "cl10k_mc5": (10_000, 100_000, 2.2, 0, 5),
}


def case_counts(name: str) -> np.ndarray:
    """Vertex degrees (out + in of the undirected graph), as huge_walk.cpp:43-46 counts them."""
    sys.path.insert(0, os.path.join(ROOT, "gdistger-re_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dgoracle
    from distger import graphgen
    n, m, beta, seed, _ = CASES[name]
    edges = graphgen.read_edges(os.path.join(HERE, "tiny200.bin")) if m == 0 else graphgen.chung_lu(n, m, beta, seed=seed)
    csr = dgoracle.Csr(edges, n, undirected=True)
    return (csr.out_deg + csr.in_deg).astype(np.uint32)


def ref_vocab(counts: np.ndarray, min_count: int):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dgoracle
    L = C.CDLL(dgoracle.REF_W2V)
    L.ref_w2v_vocab.argtypes = [C.c_void_p, C.c_uint, C.c_int, C.c_longlong] + [C.c_void_p] * 4
    n = counts.size
    ids = np.zeros(n, np.uint32)
    cn = np.zeros(n, np.int64)
    size, tw = C.c_longlong(), C.c_longlong()
    rc = L.ref_w2v_vocab(np.ascontiguousarray(counts).ctypes.data, n, min_count, n, ids.ctypes.data, cn.ctypes.data,
                         C.byref(size), C.byref(tw))
    if rc:
        raise RuntimeError("ref_w2v_vocab failed")
    k = size.value
    return ids[:k].copy(), cn[:k].copy(), tw.value


def main():
    res = {}
    for name, case in CASES.items():
        ids, cn, tw = ref_vocab(case_counts(name), case[4])
        res[name] = {"vocab_size": int(ids.size), "train_words": int(tw),
                     "ids_sha256": hashlib.sha256(ids.tobytes()).hexdigest()}
    with open(os.path.join(HERE, "w2v_vocab_ref.json"), "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
