"""Seeded inputs for the word2vec.cu kernel pin (skip_gram_kernel, cbow_kernel,
__sgNegReuse) shared by the golden-fixture generator, the GPU test that runs
the reference's own kernels, and the CPU test of the restatement.

A case is a vocabulary of counts (which fixes the unigram table), host-built
sentences (token -1 = a word the reference's batching would have skipped),
the shared negatives of __sgNegReuse, and starting rows.
"""
from __future__ import annotations

import hashlib

import numpy as np

# name: (kind, d, window, negative, alpha, vocab, sentences, seed)
# kind 0 skip_gram_kernel, 1 cbow_kernel, 2 __sgNegReuse (instantiated for d = 200 / 300 only).
CASES = {
    "sg128": (0, 128, 5, 5, 0.025, 400, 24, 11),
    "sg100": (0, 100, 3, 3, 0.025, 300, 16, 12),
    "cbow128": (1, 128, 5, 5, 0.05, 400, 24, 13),
    "cbow100": (1, 100, 4, 2, 0.05, 300, 16, 14),
    "reuse200": (2, 200, 4, 5, 0.025, 64, 8, 15),
}

TABLE_SIZE = 100_000_000  # the reference's fixed unigram-table size (word2vec.cu:66)


def make_case(name: str):
    kind, d, window, negative, alpha, vocab, n_sent, seed = CASES[name]
    rng = np.random.default_rng(seed)
    counts = np.sort(rng.zipf(1.6, vocab).clip(1, 10 ** 6).astype(np.uint32))[::-1].copy()
    lens = rng.integers(2, 28, n_sent)
    sen = rng.integers(0, vocab, int(lens.sum())).astype(np.int32)
    sen[rng.random(sen.size) < 0.04] = -1
    off = np.zeros(n_sent + 1, np.int32)
    off[1:] = np.cumsum(lens)
    # Distinct shared negatives per sentence: two warps of __sgNegReuse with the
    # same negative would race on its row.
    negs = np.stack([rng.choice(np.arange(1, vocab), negative, replace=False) for _ in range(n_sent)])
    negs = negs.astype(np.int32).reshape(-1)
    syn0 = ((rng.random((vocab, d)) - 0.5) / d).astype(np.float32)
    syn1 = (rng.standard_normal((vocab, d)) * 0.15).astype(np.float32)
    return dict(kind=kind, d=d, window=window, negative=negative, alpha=np.float32(alpha), vocab=vocab,
                counts=counts, sen=sen, off=off, negs=negs, syn0=syn0, syn1=syn1)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def unigram_table(counts: np.ndarray) -> np.ndarray:
    """word2vec.cu's InitUnigramTable (word2vec.cu:537-556) through the oracle."""
    import dgoracle
    table = np.zeros(TABLE_SIZE, np.int32)
    cn = np.ascontiguousarray(counts, dtype=np.uint32)
    dgoracle.lib().dgo_unigram_table(cn.ctypes.data, cn.size, TABLE_SIZE, table.ctypes.data)
    return table


def exp_table() -> np.ndarray:
    import dgoracle
    t = np.zeros(1001, np.float32)
    dgoracle.lib().dgo_exp_table(t.ctypes.data)
    return t


def run_reference_kernels(c: dict, table: np.ndarray, exp_tab: np.ndarray, device: int = 0):
    """The reference's kernels (oracle/_ref/libref_w2v.so) on case c, one sentence
    per launch: launch k has k + 1 blocks, the first k with empty sentences, so
    sentence k is trained by block k (LCG seeded k) with nothing racing it."""
    import ctypes as C

    import torch

    import dgoracle
    L = C.CDLL(dgoracle.REF_W2V)
    L.ref_w2v_launch.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_longlong, C.c_float] + \
        [C.c_void_p] * 10 + [C.c_int]
    L.ref_w2v_launch.restype = C.c_int
    dev = torch.device("cuda", device)
    t_table = torch.from_numpy(table).to(dev)
    t_exp = torch.from_numpy(exp_tab).to(dev)
    s0 = torch.from_numpy(c["syn0"].copy()).to(dev)
    s1 = torch.from_numpy(c["syn1"].copy()).to(dev)
    n = c["negative"]
    off = c["off"]
    for k in range(off.size - 1):
        sen = torch.from_numpy(c["sen"][off[k]:off[k + 1]].copy()).to(dev)
        so = np.zeros(k + 2, np.int32)
        so[k + 1] = off[k + 1] - off[k]
        t_so = torch.from_numpy(so).to(dev)
        ng = np.zeros((k + 1) * max(n, 1), np.int32)
        ng[k * n:(k + 1) * n] = c["negs"][k * n:(k + 1) * n]
        t_ng = torch.from_numpy(ng).to(dev)
        rc = L.ref_w2v_launch(c["kind"], c["d"], c["window"], n, 0, c["vocab"], C.c_float(c["alpha"]),
                              t_exp.data_ptr(), t_table.data_ptr(), None, None, None, s0.data_ptr(), s1.data_ptr(),
                              sen.data_ptr(), t_so.data_ptr(), t_ng.data_ptr(), k + 1)
        if rc:
            raise RuntimeError(f"reference kernel launch failed: CUDA error {rc}")
    torch.cuda.synchronize(dev)
    return s0.cpu().numpy(), s1.cpu().numpy()


def run_restatement(c: dict, table: np.ndarray, exp_tab: np.ndarray, exact_sum: int = 0):
    """dgo_w2v_sentences on case c: the restatement in the reference's own form."""
    import ctypes as C

    import dgoracle
    L = dgoracle.lib()
    cfg = dgoracle.W2vCfg(kind=c["kind"], d=c["d"], window=c["window"], negative=c["negative"],
                          alpha=float(c["alpha"]), vocab_size=c["vocab"], table_size=table.size,
                          table=table.ctypes.data, exp_table=exp_tab.ctypes.data, exact_sum=exact_sum)
    s0 = c["syn0"].copy()
    s1 = c["syn1"].copy()
    rc = L.dgo_w2v_sentences(C.byref(cfg), c["sen"].ctypes.data, c["off"].ctypes.data, c["off"].size - 1,
                             c["negs"].ctypes.data, s0.ctypes.data, s1.ctypes.data)
    if rc:
        raise RuntimeError("dgo_w2v_sentences failed")
    return s0, s1
