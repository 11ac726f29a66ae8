"""ctypes front end of the CPU checker (oracle/libdgoracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the shipped library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libdgoracle.so")
REF_WALK = os.path.join(HERE, "_ref", "ref_walk")
REF_WALK_FMA = os.path.join(HERE, "_ref", "ref_walk_fma")
REF_DSGL = os.path.join(HERE, "_ref", "ref_dsgl")
REF_W2V = os.path.join(HERE, "_ref", "libref_w2v.so")

EDGE_DTYPE = np.dtype([("src", "<u4"), ("dst", "<u4"), ("data", "<f4")])


class _Csr(C.Structure):
    _fields_ = [("v_num", C.c_uint32), ("m", C.c_uint64), ("offsets", C.POINTER(C.c_uint64)),
                ("nbr", C.POINTER(C.c_uint32)), ("data", C.POINTER(C.c_float)),
                ("out_deg", C.POINTER(C.c_uint32)), ("in_deg", C.POINTER(C.c_uint32))]


class _WalkParams(C.Structure):
    _fields_ = [("min_len", C.c_uint32), ("init_round", C.c_uint32), ("walker_num", C.c_uint32),
                ("rounds", C.c_uint32), ("seed", C.c_uint64), ("rng_mode", C.c_int),
                ("cand_cb", C.c_void_p), ("acc_cb", C.c_void_p), ("cb_ctx", C.c_void_p)]


class WalkStats(C.Structure):
    _fields_ = [("footprints", C.c_uint64), ("steps", C.c_uint64), ("draws", C.c_uint64),
                ("traces", C.c_uint64), ("pow_sq_mismatch", C.c_uint64), ("near_ties", C.c_uint64),
                ("max_len", C.c_uint32)]


class _Paths(C.Structure):
    _fields_ = [("n_walks", C.c_uint32), ("total", C.c_uint64), ("offsets", C.POINTER(C.c_uint64)),
                ("verts", C.POINTER(C.c_uint32))]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def build_ref() -> bool:
    """Compile the reference's walk engine into oracle/_ref (needs the reference tree)."""
    if os.path.exists(REF_WALK) and os.path.exists(REF_WALK_FMA):
        return True
    ref = os.environ.get("DG_REFERENCE_DIR", "")
    if not ref or not os.path.isdir(os.path.join(ref, "include")):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)
    return True


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.dgo_csr_build.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.POINTER(_Csr)]
        L.dgo_csr_free.argtypes = [C.POINTER(_Csr)]
        L.dgo_walk_round.argtypes = [C.POINTER(_Csr), C.POINTER(_WalkParams), C.c_uint32, C.c_uint32,
                                     C.POINTER(_Paths), C.POINTER(WalkStats)]
        L.dgo_paths_free.argtypes = [C.POINTER(_Paths)]
        L.dgo_write_walks.argtypes = [C.c_char_p, C.POINTER(_Paths)]
        L.dgo_relative_entropy.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        L.dgo_relative_entropy.restype = C.c_double
        L.dgo_thresholds.argtypes = [C.POINTER(_Csr), C.c_void_p]
        L.dgo_entropy_table.argtypes = [C.c_uint32, C.c_void_p]
        L.dgo_entropy_table_size.argtypes = [C.c_uint32]
        L.dgo_entropy_table_size.restype = C.c_uint64
        L.dgo_stream_new.argtypes = [C.c_uint32]
        L.dgo_stream_new.restype = C.c_void_p
        L.dgo_stream_free.argtypes = [C.c_void_p]
        L.dgo_philox.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.dgo_walk_ids.argtypes = [C.POINTER(_Csr), C.POINTER(_WalkParams), C.c_uint32, C.c_void_p, C.c_uint32,
                                   C.POINTER(_Paths), C.POINTER(WalkStats)]
        L.dgo_vocab_build.argtypes = [C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]
        L.dgo_unigram_table.argtypes = [C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p]
        L.dgo_keep_thresholds.argtypes = [C.c_void_p, C.c_uint32, C.c_float, C.c_uint64, C.c_int, C.c_void_p]
        L.dgo_init_rows.argtypes = [C.c_uint32, C.c_int, C.c_void_p]
        L.dgo_exp_table.argtypes = [C.c_void_p]
        L.dgo_sgns_plain.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]
        L.dgo_sgns_minibatch.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
        L.dgo_sgns_plain_f32.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
        L.dgo_sgns_minibatch_f32.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                             C.c_void_p, C.c_void_p]
        L.dgo_w2v_sentences.argtypes = [C.POINTER(W2vCfg), C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                        C.c_void_p, C.c_void_p]
        L.dgo_sgns_cbow_f32.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                        C.c_void_p]
        L.dgo_sgns_negshare_f32.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                            C.c_void_p, C.c_void_p]
        L.dgo_sgns_pipe.argtypes = [C.POINTER(PipeCfg), C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                    C.c_void_p]
        L.dgo_huffman.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.dgo_huffman.restype = C.c_int64
        L.dgo_dsgl_ref.argtypes = [C.POINTER(_DsglCfg), C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
        L.dgo_unigram_table_dsgl.argtypes = [C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_void_p]
        L.dgo_sgns_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_int, C.c_int64,
                                         C.c_void_p, C.c_void_p, C.c_void_p]
        L.dgo_chung_lu.argtypes = [C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_uint64, C.c_void_p]
        L.dgo_chung_lu.restype = C.c_uint64
        L.dgo_edge_data.argtypes = [C.c_uint64, C.c_uint64, C.c_int]
        L.dgo_edge_data.restype = C.c_float
        L.dgo_lp_split.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_double, C.c_uint64, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p]
        L.dgo_lp_split.restype = C.c_uint64
        _lib = L
    return _lib


def _u32(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.uint32)


class Csr:
    """Directed CSR exactly as the reference builds it for one partition."""

    def __init__(self, edges: np.ndarray, v_num: int, undirected: bool = True):
        edges = np.ascontiguousarray(edges, dtype=EDGE_DTYPE)
        self._c = _Csr()
        rc = lib().dgo_csr_build(edges.ctypes.data, edges.size, v_num, int(undirected), C.byref(self._c))
        if rc:
            raise ValueError(f"dgo_csr_build failed ({rc})")
        m = self._c.m
        self.v_num = v_num
        self.m = m
        self.offsets = np.ctypeslib.as_array(self._c.offsets, shape=(v_num + 1,)).copy()
        self.nbr = _u32(self._c.nbr, m)
        self.data = np.ctypeslib.as_array(self._c.data, shape=(m,)).copy() if m else np.zeros(0, np.float32)
        self.out_deg = _u32(self._c.out_deg, v_num)
        self.in_deg = _u32(self._c.in_deg, v_num)

    def thresholds(self) -> np.ndarray:
        out = np.empty(self.m, dtype=np.uint32)
        lib().dgo_thresholds(C.byref(self._c), out.ctypes.data)
        return out

    def __del__(self):
        try:
            lib().dgo_csr_free(C.byref(self._c))
        except Exception:
            pass


def walk_rounds(csr: Csr, walker_num: int, min_len: int = 20, init_round: int = 5, rounds: int = 30,
                seed: int = 0, stream_seed: int | None = None, first_round: int = 1,
                round_walkers=None):
    """Run rounds first_round..rounds as internal_random_walk does (walk.hpp:609-782).

    Returns (list of (offsets, verts) per round, WalkStats).  With stream_seed set,
    the reference's mt19937/rand() streams are consumed in one-worker order
    instead of Philox.
    """
    L = lib()
    p = _WalkParams(min_len=min_len, init_round=init_round, walker_num=walker_num, rounds=rounds,
                    seed=seed, rng_mode=0)
    ctx = None
    if stream_seed is not None:
        ctx = L.dgo_stream_new(stream_seed)
        p.rng_mode = 1
        p.cand_cb = C.cast(L.dgo_stream_cand, C.c_void_p).value
        p.acc_cb = C.cast(L.dgo_stream_acc, C.c_void_p).value
        p.cb_ctx = ctx
    stats = WalkStats()
    out = []
    try:
        for r in range(first_round, rounds + 1):
            n = round_walkers(r) if round_walkers else (walker_num * init_round if r == 1 else walker_num)
            paths = _Paths()
            rc = L.dgo_walk_round(C.byref(csr._c), C.byref(p), r, n, C.byref(paths), C.byref(stats))
            if rc:
                raise RuntimeError(f"dgo_walk_round failed ({rc})")
            offs = np.ctypeslib.as_array(paths.offsets, shape=(n + 1,)).copy()
            verts = _u32(paths.verts, paths.total)
            L.dgo_paths_free(C.byref(paths))
            out.append((offs, verts))
    finally:
        if ctx is not None:
            L.dgo_stream_free(ctx)
    return out, stats


def walk_ids(csr: Csr, ids, round_index: int, min_len: int = 20, seed: int = 0):
    """Philox-mode walks of the given walker ids of one round: (offsets, verts)."""
    L = lib()
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    p = _WalkParams(min_len=min_len, init_round=1, walker_num=1, rounds=round_index, seed=seed, rng_mode=0)
    paths = _Paths()
    stats = WalkStats()
    rc = L.dgo_walk_ids(C.byref(csr._c), C.byref(p), round_index, ids.ctypes.data, ids.size, C.byref(paths),
                        C.byref(stats))
    if rc:
        raise RuntimeError(f"dgo_walk_ids failed ({rc})")
    offs = np.ctypeslib.as_array(paths.offsets, shape=(ids.size + 1,)).copy()
    verts = _u32(paths.verts, paths.total)
    L.dgo_paths_free(C.byref(paths))
    return offs, verts


def walk_text(offsets: np.ndarray, verts: np.ndarray) -> bytes:
    """Walk file bytes: " %u" per vertex, "\\n" per walk (path.hpp:92,108)."""
    parts = []
    for w in range(offsets.size - 1):
        seg = verts[offsets[w]:offsets[w + 1]]
        parts.append("".join(" %d" % x for x in seg.tolist()) + "\n")
    return "".join(parts).encode()


def relative_entropy(out_deg: np.ndarray, freq: np.ndarray) -> float:
    out_deg = np.ascontiguousarray(out_deg, dtype=np.uint32)
    freq = np.ascontiguousarray(freq, dtype=np.uint32)
    return lib().dgo_relative_entropy(out_deg.ctypes.data, freq.ctypes.data, out_deg.size)


def philox(ctr, key) -> list:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().dgo_philox(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    return [int(x) for x in out]


def load_golden(path: str):
    z = np.load(path)
    rounds = []
    r = 1
    while f"offsets_{r}" in z:
        rounds.append((z[f"offsets_{r}"], z[f"verts_{r}"]))
        r += 1
    return rounds, z["abs_delta_h"], z["meta"]


class _SgnsCfg(C.Structure):
    _fields_ = [("d", C.c_int), ("window", C.c_int), ("negative", C.c_int), ("alpha", C.c_double),
                ("seed", C.c_uint64), ("pass_", C.c_uint32), ("vocab_size", C.c_uint32),
                ("table_size", C.c_uint64), ("table", C.c_void_p), ("keep_thr", C.c_void_p),
                ("v2w", C.c_void_p), ("exp_table", C.c_void_p), ("hs", C.c_int), ("hs_off", C.c_void_p),
                ("hs_point", C.c_void_p), ("hs_code", C.c_void_p)]


class SgnsStats(C.Structure):
    _fields_ = [("words", C.c_uint64), ("trained", C.c_uint64), ("pairs", C.c_uint64)]


class W2vCfg(C.Structure):
    _fields_ = [("kind", C.c_int), ("d", C.c_int), ("window", C.c_int), ("negative", C.c_int),
                ("alpha", C.c_float), ("vocab_size", C.c_uint32), ("table_size", C.c_uint64),
                ("table", C.c_void_p), ("exp_table", C.c_void_p), ("exact_sum", C.c_int), ("hs", C.c_int),
                ("hs_off", C.c_void_p), ("hs_point", C.c_void_p), ("hs_code", C.c_void_p)]


class PipeCfg(C.Structure):
    _fields_ = [("d", C.c_int), ("window", C.c_int), ("negative", C.c_int), ("stages", C.c_int), ("bf16", C.c_int),
                ("alpha", C.c_float), ("seed", C.c_uint64), ("seed_lo", C.c_uint32), ("pass_", C.c_uint32),
                ("vocab_size", C.c_uint32), ("n_master", C.c_uint32), ("table_size", C.c_uint64),
                ("table", C.c_void_p), ("keep_thr", C.c_void_p), ("v2w", C.c_void_p), ("exp_table", C.c_void_p)]


def sgns_pipe(tables: dict, rows_in, rows_out, offsets, verts, size: int, window: int, negative: int, alpha: float,
              seed: int, pass_: int, stages: int = 2, bf16: bool = False, n_master: int = 0):
    """The one-warp staged-rows kernel modelled on the CPU (dgo_sgns_pipe); rows are
    updated in place (C-contiguous FP32 arrays in vocabulary order)."""
    t = tables
    assert rows_in.flags.c_contiguous and rows_out.flags.c_contiguous
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    verts = np.ascontiguousarray(verts, dtype=np.uint32)
    cfg = PipeCfg(d=size, window=window, negative=negative, stages=stages, bf16=int(bf16), alpha=alpha,
                  seed=seed, seed_lo=seed & 0xFFFFFFFF, pass_=pass_, vocab_size=t["keep_thr"].size,
                  n_master=n_master, table_size=t["table"].size, table=t["table"].ctypes.data,
                  keep_thr=t["keep_thr"].ctypes.data, v2w=t["v2w"].ctypes.data, exp_table=t["exp_table"].ctypes.data)
    st = SgnsStats()
    rc = lib().dgo_sgns_pipe(C.byref(cfg), offsets.ctypes.data, verts.ctypes.data, offsets.size - 1,
                             rows_in.ctypes.data, rows_out.ctypes.data, C.byref(st))
    if rc:
        raise RuntimeError(f"dgo_sgns_pipe failed ({rc})")
    return st


class _DsglCfg(C.Structure):
    _fields_ = [("d", C.c_int), ("window", C.c_int), ("negative", C.c_int), ("iter", C.c_int),
                ("sample", C.c_float), ("alpha", C.c_float), ("train_words", C.c_uint64),
                ("vocab_size", C.c_uint32), ("table_size", C.c_uint64), ("table", C.c_void_p),
                ("ran", C.c_void_p), ("v2w", C.c_void_p), ("exp_table", C.c_void_p), ("device_order", C.c_int)]


def huffman(cn: np.ndarray):
    """word2vec's Huffman coding restated (dgo_huffman): (off, point, code) in the
    kernels' prefix layout for counts in vocabulary order."""
    cn = np.ascontiguousarray(cn, dtype=np.uint64)
    n = cn.size
    off = np.zeros(n + 1, np.int32)
    point = np.zeros(n * 40, np.int32)
    code = np.zeros(n * 40, np.int8)
    total = lib().dgo_huffman(cn.ctypes.data, n, off.ctypes.data, point.ctypes.data, code.ctypes.data)
    if total < 0:
        raise ValueError("Huffman code longer than 40 bits, or fewer than 2 words")
    return off, point[:total].copy(), code[:total].copy()


def ref_huffman(cn: np.ndarray):
    """The reference's own CreateBinaryTree (oracle/_ref/libref_w2v.so, host code), in
    the same prefix layout."""
    L = C.CDLL(REF_W2V)
    L.ref_w2v_huffman.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p]
    cn = np.ascontiguousarray(cn, dtype=np.int64)
    n = cn.size
    cl = np.zeros(n, np.int32)
    point = np.zeros(n * 40, np.int32)
    code = np.zeros(n * 40, np.int8)
    L.ref_w2v_huffman(cn.ctypes.data, n, cl.ctypes.data, point.ctypes.data, code.ctypes.data)
    off = np.zeros(n + 1, np.int32)
    off[1:] = np.cumsum(cl)
    p = np.concatenate([point[a * 40:a * 40 + cl[a]] for a in range(n)]) if n else np.zeros(0, np.int32)
    c = np.concatenate([code[a * 40:a * 40 + cl[a]] for a in range(n)]) if n else np.zeros(0, np.int8)
    return off, p.astype(np.int32), c.astype(np.int8)


def dsgl_vocab(counts: np.ndarray):
    """dsgl's vocabulary (dsgl.hpp:355-378): vertices sorted by count, descending.
    Only counts without ties give a unique order (std::sort is not stable)."""
    counts = np.asarray(counts, dtype=np.int64)
    order = np.argsort(-counts, kind="stable").astype(np.uint32)
    v2w = np.empty(counts.size, np.int32)
    v2w[order] = np.arange(counts.size, dtype=np.int32)
    return order, v2w


def dsgl_ref(counts: np.ndarray, corpus: np.ndarray, size: int, window: int, negative: int, sample: float,
             alpha: float, iterations: int = 1, table_size: int = 100_000_000, device_order: bool = False):
    """dsgl's trainer restated in its own random stream and GEMM order (dgo_dsgl_ref);
    device_order=True evaluates each step in the device kernel's order instead.

    counts: vertex_cn (int per vertex id); corpus: vertex ids with -1 after every
    walk.  Returns (vocabulary ids, Wih, Woh, final alpha) in vocabulary order."""
    L = lib()
    counts = np.ascontiguousarray(counts, dtype=np.int32)
    corpus = np.ascontiguousarray(corpus, dtype=np.int32)
    ids, v2w = dsgl_vocab(counts)
    vs = counts.size
    cn_sorted = np.ascontiguousarray(counts[ids].astype(np.uint32))
    train_words = int(counts.astype(np.int64).sum())
    table = np.zeros(table_size, np.int32)
    L.dgo_unigram_table_dsgl(cn_sorted.ctypes.data, vs, table_size, 2, table.ctypes.data)
    # dsgl.hpp:933-935 reads the count at (*cn_vocab)[w] with w a vocabulary
    # index, i.e. the count of VERTEX w, not of the word w.
    st = np.float32(sample) * np.float32(train_words)
    with np.errstate(divide="ignore"):
        ratio = (st / counts.astype(np.float32)).astype(np.float32)
    ran = (np.sqrt(ratio) + ratio).astype(np.float32)
    exp_table = np.zeros(1001, np.float32)
    L.dgo_exp_table(exp_table.ctypes.data)
    wih = np.zeros(vs * size, np.float32)
    L.dgo_init_rows(vs, size, wih.ctypes.data)
    woh = np.zeros(vs * size, np.float32)
    cfg = _DsglCfg(d=size, window=window, negative=negative, iter=iterations, sample=sample, alpha=alpha,
                   train_words=train_words, vocab_size=vs, table_size=table_size, table=table.ctypes.data,
                   ran=ran.ctypes.data, v2w=v2w.ctypes.data, exp_table=exp_table.ctypes.data,
                   device_order=int(device_order))
    a_out = C.c_float()
    stats = SgnsStats()
    rc = L.dgo_dsgl_ref(C.byref(cfg), corpus.ctypes.data, corpus.size, wih.ctypes.data, woh.ctypes.data,
                        C.byref(a_out), C.byref(stats))
    if rc:
        raise RuntimeError("dgo_dsgl_ref failed")
    return ids, wih.reshape(vs, size), woh.reshape(vs, size), a_out.value


def write_dsgl_corpus(path: str, counts: np.ndarray, corpus: np.ndarray) -> None:
    counts = np.ascontiguousarray(counts, dtype=np.int32)
    corpus = np.ascontiguousarray(corpus, dtype=np.int32)
    with open(path, "wb") as f:
        f.write(np.uint32(counts.size).tobytes())
        f.write(counts.tobytes())
        f.write(np.uint64(corpus.size).tobytes())
        f.write(corpus.tobytes())


def read_dsgl_dump(path: str):
    raw = open(path, "rb").read()
    vs, d = np.frombuffer(raw[:16], np.uint64)
    vs, d = int(vs), int(d)
    o = 16
    ids = np.frombuffer(raw[o:o + 4 * vs], np.uint32).copy(); o += 4 * vs
    wih = np.frombuffer(raw[o:o + 4 * vs * d], np.float32).reshape(vs, d).copy(); o += 4 * vs * d
    woh = np.frombuffer(raw[o:o + 4 * vs * d], np.float32).reshape(vs, d).copy(); o += 4 * vs * d
    alpha = float(np.frombuffer(raw[o:o + 4], np.float32)[0])
    return ids, wih, woh, alpha


def run_ref_dsgl(workdir: str, counts: np.ndarray, corpus: np.ndarray, size: int, window: int, negative: int,
                 sample: float, alpha: float, iterations: int = 1, sync_period: float = 5.0):
    """Runs the reference's own dsgl (oracle/_ref/ref_dsgl, one compute thread)."""
    cpath = os.path.join(workdir, "corpus.bin")
    dpath = os.path.join(workdir, "dump.bin")
    write_dsgl_corpus(cpath, counts, corpus)
    cmd = [REF_DSGL, "--corpus", cpath, "--dump", dpath, "-size", str(size), "-window", str(window),
           "-negative", str(negative), "-sample", repr(float(sample)), "-alpha", repr(float(alpha)),
           "-iter", str(iterations), "-threads", "2", "-sync-period", str(sync_period), "-min-count", "0",
           "-debug", "0", "-eoutput", os.path.join(workdir, "emb.txt")]
    subprocess.run(cmd, check=True, capture_output=True)
    return read_dsgl_dump(dpath)


class Sgns:
    """FP64 SGNS checker: vocabulary, tables and both update rules."""

    def __init__(self, counts: np.ndarray, size: int = 128, window: int = 10, negative: int = 5,
                 sample: float = 1e-3, alpha: float = 0.025, min_count: int = 0, seed: int = 0,
                 table_size: int = 100_000_000, dsgl_form: bool = False, hs: bool = False):
        L = lib()
        counts = np.ascontiguousarray(counts, dtype=np.uint32)
        v_num = counts.size
        self.vocab_ids = np.zeros(v_num, np.uint32)
        self.vocab_cn = np.zeros(v_num, np.uint32)
        self.v2w = np.zeros(v_num, np.int32)
        vs = C.c_uint32()
        tw = C.c_uint64()
        rc = L.dgo_vocab_build(counts.ctypes.data, v_num, min_count, self.vocab_ids.ctypes.data,
                               self.vocab_cn.ctypes.data, self.v2w.ctypes.data, C.byref(vs), C.byref(tw))
        if rc:
            raise RuntimeError("vocab build failed")
        self.vocab_size = vs.value
        self.train_words = tw.value
        self.vocab_ids = self.vocab_ids[:self.vocab_size]
        self.vocab_cn = self.vocab_cn[:self.vocab_size]
        self.table = np.zeros(table_size, np.int32)
        L.dgo_unigram_table(self.vocab_cn.ctypes.data, self.vocab_size, table_size, self.table.ctypes.data)
        self.keep_thr = np.zeros(self.vocab_size, np.uint32)
        L.dgo_keep_thresholds(self.vocab_cn.ctypes.data, self.vocab_size, C.c_float(sample), tw.value,
                              int(dsgl_form), self.keep_thr.ctypes.data)
        self.exp_table = np.zeros(1001, np.float32)
        L.dgo_exp_table(self.exp_table.ctypes.data)
        init = np.zeros(self.vocab_size * size, np.float32)
        L.dgo_init_rows(self.vocab_size, size, init.ctypes.data)
        self.syn0 = init.astype(np.float64).reshape(self.vocab_size, size)
        self.syn1 = np.zeros((self.vocab_size, size), np.float64)
        # FP32 rows updated in the device kernels' operation order.
        self.syn0_f32 = init.reshape(self.vocab_size, size).copy()
        self.syn1_f32 = np.zeros((self.vocab_size, size), np.float32)
        self.stats_f32 = SgnsStats()
        self.size, self.window, self.negative, self.alpha, self.seed = size, window, negative, alpha, seed
        self.hs = bool(hs)
        if self.hs:
            self.hs_off, self.hs_point, self.hs_code = huffman(self.vocab_cn)
        self.pass_ = 0
        self.stats = SgnsStats()

    def _cfg(self, alpha):
        return _SgnsCfg(d=self.size, window=self.window, negative=self.negative,
                        alpha=self.alpha if alpha is None else alpha, seed=self.seed, pass_=self.pass_,
                        vocab_size=self.vocab_size, table_size=self.table.size, table=self.table.ctypes.data,
                        keep_thr=self.keep_thr.ctypes.data, v2w=self.v2w.ctypes.data,
                        exp_table=self.exp_table.ctypes.data, hs=int(self.hs),
                        hs_off=self.hs_off.ctypes.data if self.hs else None,
                        hs_point=self.hs_point.ctypes.data if self.hs else None,
                        hs_code=self.hs_code.ctypes.data if self.hs else None)

    def train(self, offsets: np.ndarray, verts: np.ndarray, minibatch: bool = False, alpha=None,
              rule: str = "plain"):
        """One pass over the walks.  rule: "plain" (skip-gram, FP64 + FP32),
        "minibatch" (dsgl, FP64 + FP32; also selected by minibatch=True), "cbow" or
        "negshare" (FP32 rows only, syn0_f32 / syn1_f32)."""
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        verts = np.ascontiguousarray(verts, dtype=np.uint32)
        cfg = self._cfg(alpha)
        n = offsets.size - 1
        L = lib()
        if rule in ("cbow", "negshare"):
            fn = L.dgo_sgns_cbow_f32 if rule == "cbow" else L.dgo_sgns_negshare_f32
            rc = fn(C.byref(cfg), offsets.ctypes.data, verts.ctypes.data, n, self.syn0_f32.ctypes.data,
                    self.syn1_f32.ctypes.data, C.byref(self.stats_f32))
        elif minibatch or rule == "minibatch":
            rc = L.dgo_sgns_minibatch(C.byref(cfg), offsets.ctypes.data, verts.ctypes.data, n,
                                      self.syn0.ctypes.data, self.syn1.ctypes.data, C.byref(self.stats))
            rc |= L.dgo_sgns_minibatch_f32(C.byref(cfg), offsets.ctypes.data, verts.ctypes.data, n,
                                           self.syn0_f32.ctypes.data, self.syn1_f32.ctypes.data,
                                           C.byref(self.stats_f32))
        else:
            rc = L.dgo_sgns_plain(C.byref(cfg), offsets.ctypes.data, verts.ctypes.data, n, None,
                                  self.syn0.ctypes.data, self.syn1.ctypes.data, C.byref(self.stats))
            rc |= L.dgo_sgns_plain_f32(C.byref(cfg), offsets.ctypes.data, verts.ctypes.data, n,
                                       self.syn0_f32.ctypes.data, self.syn1_f32.ctypes.data,
                                       C.byref(self.stats_f32))
        if rc:
            raise RuntimeError("sgns oracle failed")
        self.pass_ += 1


def entropy_table(max_sn: int) -> np.ndarray:
    n = lib().dgo_entropy_table_size(max_sn)
    out = np.empty(n, dtype=np.float64)
    lib().dgo_entropy_table(max_sn, out.ctypes.data)
    return out


def sgns_loss_grad(in_rows: np.ndarray, out_rows: np.ndarray, inputs, outputs, negatives, batch: int,
                   negative: int, grad: bool = True, only=None):
    """FP64 SGNS loss (and gradient) over explicit minibatches (dg_oracle_adjoint.c).
    only = (table, row) restricts the sum to the pairs whose terms depend on that row."""
    a = np.ascontiguousarray(in_rows, dtype=np.float64)
    b = np.ascontiguousarray(out_rows, dtype=np.float64)
    vocab, d = a.shape
    inp = np.ascontiguousarray(inputs, dtype=np.uint32)
    outp = np.ascontiguousarray(outputs, dtype=np.uint32)
    neg = np.ascontiguousarray(negatives, dtype=np.uint32)
    loss = C.c_double()
    gi = np.zeros((vocab, d)) if grad else None
    go = np.zeros((vocab, d)) if grad else None
    table, row = only if only is not None else (0, -1)
    rc = lib().dgo_sgns_loss_grad(a.ctypes.data, b.ctypes.data, d, vocab, inp.ctypes.data, outp.ctypes.data,
                                  neg.ctypes.data if neg.size else None, inp.size, batch, negative, table, row,
                                  C.byref(loss), gi.ctypes.data if grad else None,
                                  go.ctypes.data if grad else None)
    if rc:
        raise RuntimeError("dgo_sgns_loss_grad failed")
    return loss.value, gi, go


def chung_lu_keys(n: int, m: int, beta: float, max_degree: float, seed: int) -> np.ndarray:
    """Unique undirected pair keys (lo << 32 | hi) of the device generator, restated (dg_oracle_gen.c)."""
    keys = np.zeros(m + n, np.uint64)
    e = lib().dgo_chung_lu(n, m, beta, max_degree or 0.0, seed, keys.ctypes.data)
    return keys[:e].copy()


def edge_data(keys: np.ndarray, seed: int, weighted: bool) -> np.ndarray:
    L = lib()
    return np.array([L.dgo_edge_data(int(k), seed, int(weighted)) for k in keys.tolist()], np.float32)


def lp_split(keys: np.ndarray, v_num: int, frac: float, seed: int):
    """(kept keys, positives (u, v), negatives (u, v)) of the device split, restated."""
    k = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    n = k.size
    pu, pv, nu, nv = (np.zeros(max(n, 1), np.uint32) for _ in range(4))
    npos = C.c_uint64()
    nk = lib().dgo_lp_split(k.ctypes.data, n, v_num, frac, seed, pu.ctypes.data, pv.ctypes.data, nu.ctypes.data,
                            nv.ctypes.data, C.byref(npos))
    p = npos.value
    return k[:nk], (pu[:p], pv[:p]), (nu[:p], nv[:p])


def common_neighbours(src, dst, v_num: int, undirected: bool = True) -> np.ndarray:
    """Common-neighbour counts of the reference's gcn tool (src/tools/gcn.cpp:249-373), restated:
    rows sorted by neighbour with duplicates (130-137); for edge (s, d) the elements of the shorter
    row (N(s) on a tie, 166-172) found in the other row, with the shorter row's multiplicity; less
    one if the first is s or d, and, when more than one remains, less one per later element that
    repeats its predecessor or is s or d (327-343); a repeated pair reports its first occurrence's
    value (305-310, 348-352).  An empty row gives 0."""
    import bisect
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    a = np.concatenate([src, dst]) if undirected else src
    b = np.concatenate([dst, src]) if undirected else dst
    order = np.lexsort((b, a))
    a, b = a[order], b[order]
    offs = np.zeros(v_num + 1, np.int64)
    np.add.at(offs, a + 1, 1)
    offs = np.cumsum(offs)
    rows = b.tolist()
    seen = {}
    out = np.zeros(src.size, np.int32)
    for e, (s, d) in enumerate(zip(src.tolist(), dst.tolist())):
        key = (min(s, d), max(s, d))
        if key not in seen:
            r1 = rows[offs[s]:offs[s + 1]]
            r2 = rows[offs[d]:offs[d + 1]]
            lg, sh = (r1, r2) if len(r1) > len(r2) else (r2, r1)
            inter = []
            if lg and sh:
                for x in sh:
                    i = bisect.bisect_left(lg, x)
                    if i < len(lg) and lg[i] == x:
                        inter.append(x)
            cn = len(inter)
            if cn > 0:
                if inter[0] in (s, d):
                    cn -= 1
                if cn > 1:
                    for i in range(1, len(inter)):
                        if inter[i] == inter[i - 1] or inter[i] in (s, d):
                            cn -= 1
            seen[key] = cn
        out[e] = seen[key]
    return out
