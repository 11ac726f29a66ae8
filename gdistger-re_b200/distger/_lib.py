"""ctypes binding of the distger C ABI (include/distger.h, libdistger.so).

The CUDA library is the only compute path: if libdistger.so is missing or
cannot be loaded, every call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libdistger.so")
CSRC = os.path.join(PKG_DIR, "csrc")

DG_OK = 0
ERRORS = {-1: "DG_ERR_ARG", -2: "DG_ERR_IO", -3: "DG_ERR_CUDA", -4: "DG_ERR_NOMEM", -5: "DG_ERR_OVERFLOW",
          -6: "DG_ERR_STATE"}


class DistgerError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class GraphInfo(C.Structure):
    _fields_ = [("v_num", C.c_uint32), ("m", C.c_uint64), ("device_bytes", C.c_uint64),
                ("threshold_ms", C.c_double)]


class WalkParams(C.Structure):
    _fields_ = [("min_len", C.c_uint32), ("init_round", C.c_uint32), ("walker_num", C.c_uint32),
                ("max_len", C.c_uint32), ("seed", C.c_uint64)]


class RoundInfo(C.Structure):
    _fields_ = [("n_walks", C.c_uint32), ("footprints", C.c_uint64), ("steps", C.c_uint64),
                ("draws", C.c_uint64), ("traces", C.c_uint64), ("max_len", C.c_uint32),
                ("walk_ms", C.c_double), ("relative_entropy", C.c_double), ("delta_h", C.c_double)]


class SgnsParams(C.Structure):
    _fields_ = [("size", C.c_int), ("window", C.c_int), ("negative", C.c_int), ("batch_size", C.c_int),
                ("sample", C.c_float), ("alpha", C.c_float), ("iter", C.c_int), ("min_count", C.c_int),
                ("mode", C.c_int), ("deterministic", C.c_int), ("seed", C.c_uint64),
                ("table_size", C.c_uint64), ("master_rows", C.c_uint32), ("workers", C.c_uint32),
                ("hs", C.c_int)]


class TrainInfo(C.Structure):
    _fields_ = [("words", C.c_uint64), ("trained", C.c_uint64), ("pairs", C.c_uint64),
                ("train_ms", C.c_double), ("rows", C.c_uint64)]


class PipelineInfo(C.Structure):
    _fields_ = [("walk", RoundInfo), ("train", TrainInfo), ("total_ms", C.c_double)]


class MinibatchArgs(C.Structure):
    """dg_sgns_minibatch_args: device pointers for the allocation-free trainer."""
    _fields_ = [("verts", C.c_void_p), ("offsets", C.c_void_p), ("n_walks", C.c_uint32),
                ("v2w", C.c_void_p), ("keep_thr", C.c_void_p), ("table", C.c_void_p),
                ("table_size", C.c_uint64), ("exp_table", C.c_void_p), ("vocab_size", C.c_uint32),
                ("in_bf16", C.c_void_p), ("out_bf16", C.c_void_p), ("in_master", C.c_void_p),
                ("out_master", C.c_void_p), ("n_master", C.c_uint32), ("size", C.c_int), ("window", C.c_int),
                ("negative", C.c_int), ("alpha", C.c_float), ("seed", C.c_uint64), ("pass_", C.c_uint32),
                ("deterministic", C.c_int), ("workers", C.c_uint32)]


class SgnsInfo(C.Structure):
    _fields_ = [("vocab_size", C.c_uint32), ("master_rows", C.c_uint32), ("workers", C.c_uint32),
                ("train_words", C.c_uint64),
                ("table_size", C.c_uint64), ("device_bytes", C.c_uint64), ("bf_staged", C.c_int32)]


class SgnsPairs(C.Structure):
    """dg_sgns_pairs: explicit shared-negative minibatches (host pointers)."""
    _fields_ = [("inputs", C.c_void_p), ("outputs", C.c_void_p), ("negatives", C.c_void_p),
                ("n_pairs", C.c_uint64), ("batch", C.c_uint32), ("negative", C.c_int)]


class TuneInfo(C.Structure):
    """dg_tune_info: the launch shapes timed by an autotune call and the one kept."""
    _fields_ = [("n_candidates", C.c_int), ("chosen", C.c_int), ("shape", (C.c_int * 3) * 16),
                ("ms", C.c_double * 16)]

    def as_dict(self) -> dict:
        n = min(self.n_candidates, 16)
        return {"chosen": self.chosen, "candidates": [{"shape": [self.shape[k][0], self.shape[k][1], self.shape[k][2]],
                                                       "ms": self.ms[k]} for k in range(n)]}


_P = C.c_void_p
_SIGS = {
    "dg_last_error": ([], C.c_char_p),
    "dg_version": ([], C.c_char_p),
    "dg_graph_create": ([C.c_char_p, C.c_uint32, C.c_int, C.c_int, C.POINTER(_P)], C.c_int),
    "dg_graph_create_from_edges": ([_P, C.c_uint64, C.c_uint32, C.c_int, C.c_int, C.POINTER(_P)], C.c_int),
    "dg_graph_free": ([_P], None),
    "dg_graph_get_info": ([_P, C.POINTER(GraphInfo)], C.c_int),
    "dg_graph_copy_csr": ([_P, _P, _P, _P, _P, _P], C.c_int),
    "dg_graph_copy_visits": ([_P, _P], C.c_int),
    "dg_walk_run_round": ([_P, C.POINTER(WalkParams), C.c_uint32, C.c_uint32, C.POINTER(_P)], C.c_int),
    "dg_paths_get_info": ([_P, C.POINTER(RoundInfo)], C.c_int),
    "dg_paths_copy": ([_P, _P, _P], C.c_int),
    "dg_paths_write_text": ([_P, C.c_char_p], C.c_int),
    "dg_paths_free": ([_P], None),
    "dg_sgns_create": ([C.POINTER(SgnsParams), C.c_uint32, _P, C.c_int, C.POINTER(_P)], C.c_int),
    "dg_sgns_free": ([_P], None),
    "dg_sgns_train_paths": ([_P, _P, C.c_float, C.POINTER(TrainInfo)], C.c_int),
    "dg_sgns_train_host": ([_P, _P, C.c_uint32, _P, C.c_float, C.POINTER(TrainInfo)], C.c_int),
    "dg_sgns_copy_embedding": ([_P, _P, _P, C.POINTER(C.c_uint32)], C.c_int),
    "dg_sgns_copy_output": ([_P, _P], C.c_int),
    "dg_sgns_set_rows": ([_P, _P, _P], C.c_int),
    "dg_sgns_write_embedding": ([_P, C.c_char_p], C.c_int),
    "dg_sgns_copy_tables": ([_P, _P, _P, _P, _P], C.c_int),
    "dg_sgns_get_info": ([_P, C.POINTER(SgnsInfo)], C.c_int),
    "dg_pipeline_round": ([_P, _P, C.POINTER(WalkParams), C.c_uint32, C.c_uint32, C.c_float,
                           C.POINTER(PipelineInfo), C.POINTER(_P)], C.c_int),
    "dg_launch_count": ([], C.c_uint64),
    "dg_sgns_minibatch_train_noalloc": ([C.POINTER(MinibatchArgs), _P, C.POINTER(TrainInfo)], C.c_int),
    "dg_sgns_loss_grad": ([_P, C.POINTER(SgnsPairs), C.POINTER(C.c_double), _P, _P], C.c_int),
    "dg_sgns_adjoint_step": ([_P, C.POINTER(SgnsPairs), C.c_float, C.POINTER(C.c_double)], C.c_int),
    "dg_walk_autotune": ([_P, C.POINTER(WalkParams), C.c_uint32, C.c_uint32, C.POINTER(TuneInfo)], C.c_int),
    "dg_walk_set_shape": ([_P, C.c_int], C.c_int),
    "dg_sgns_autotune": ([_P, _P, C.POINTER(TuneInfo)], C.c_int),
    "dg_sgns_set_shape": ([_P, C.c_int], C.c_int),
    "dg_edges_chung_lu": ([_P, C.c_int, C.POINTER(_P)], C.c_int),
    "dg_edges_get_info": ([_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)], C.c_int),
    "dg_edges_copy": ([_P, _P, _P, _P], C.c_int),
    "dg_edges_free": ([_P], None),
    "dg_edges_split": ([_P, C.c_double, C.c_uint64, C.POINTER(_P)], C.c_int),
    "dg_lp_pairs_get_info": ([_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)], C.c_int),
    "dg_lp_pairs_copy": ([_P, _P, _P, _P], C.c_int),
    "dg_lp_pairs_free": ([_P], None),
    "dg_graph_create_from_device_edges": ([_P, C.POINTER(_P)], C.c_int),
    "dg_lp_auc": ([_P, _P, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
    "dg_common_neighbours": ([_P, _P, C.c_uint64, C.c_uint32, C.c_int, C.c_int, _P], C.c_int),
}

_lib = None


def build() -> None:
    """Compile the CUDA sources for sm_100a into gdistger-re_b200/libdistger.so."""
    subprocess.run(["make", "-s", "-C", CSRC], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is not built; run distger.build() (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != DG_OK:
        raise DistgerError(rc, lib().dg_last_error().decode(errors="replace"))
