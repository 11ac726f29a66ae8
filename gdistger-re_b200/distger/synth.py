"""Synthetic graphs, the link-prediction split and AUC scoring on the device.

Host-side mirror of the dg_edges_* / dg_lp_* entry points (include/distger.h):
`EdgeList.chung_lu` generates a Chung-Lu graph in HBM, `split` holds out edges
and non-edges with the rule of src/tools/gtrain.cpp:226-386 in its parallel
form, `graph` builds the undirected CSR on the device, and `LinkPairs.auc`
scores a trainer's input embedding.  For graphs that fit host tools the numpy
generator (graphgen) and scorer (lp) do the same jobs on the CPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np


from ._lib import check, lib
from .walk import Graph

class ChungLuParams(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("beta", C.c_double), ("max_degree", C.c_double),
                ("seed", C.c_uint64), ("weighted", C.c_int)]


def _L():
    return lib()


class LinkPairs:
    """Held-out edges (label 1) followed by as many non-edges (label 0), on the device."""

    def __init__(self, handle, device: int):
        self._h = handle
        self.device = device
        a, b = C.c_uint64(), C.c_uint64()
        check(_L().dg_lp_pairs_get_info(handle, C.byref(a), C.byref(b)))
        self.n_pos, self.n_neg = a.value, b.value

    def to_numpy(self):
        n = self.n_pos + self.n_neg
        u, v, lab = np.empty(n, np.uint32), np.empty(n, np.uint32), np.empty(n, np.uint8)
        if n:
            check(_L().dg_lp_pairs_copy(self._h, u.ctypes.data, v.ctypes.data, lab.ctypes.data))
        return u, v, lab

    def auc(self, sgns) -> dict:
        a, c = C.c_double(), C.c_double()
        check(_L().dg_lp_auc(sgns.handle, self._h, C.byref(a), C.byref(c)))
        return {"auc": a.value, "auc_cosine": c.value}

    def close(self):
        if getattr(self, "_h", None):
            _L().dg_lp_pairs_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class EdgeList:
    """Unique undirected pairs (src < dst, ascending) resident on the device."""

    def __init__(self, handle, device: int):
        self._h = handle
        self.device = device
        self._info()

    def _info(self):
        v, n = C.c_uint32(), C.c_uint64()
        check(_L().dg_edges_get_info(self._h, C.byref(v), C.byref(n)))
        self.v_num, self.n = v.value, n.value

    @classmethod
    def chung_lu(cls, n: int, m: int, beta: float, seed: int = 0, max_degree: float | None = None,
                 weighted: bool = True, device: int = 0) -> "EdgeList":
        p = ChungLuParams(n=n, m=m, beta=beta, max_degree=max_degree or 0.0, seed=seed, weighted=int(weighted))
        h = C.c_void_p()
        check(_L().dg_edges_chung_lu(C.byref(p), device, C.byref(h)))
        return cls(h, device)

    def to_numpy(self):
        src, dst, data = np.empty(self.n, np.uint32), np.empty(self.n, np.uint32), np.empty(self.n, np.float32)
        if self.n:
            check(_L().dg_edges_copy(self._h, src.ctypes.data, dst.ctypes.data, data.ctypes.data))
        return src, dst, data

    def split(self, frac: float = 0.1, seed: int = 2) -> LinkPairs:
        h = C.c_void_p()
        check(_L().dg_edges_split(self._h, frac, seed, C.byref(h)))
        self._info()
        return LinkPairs(h, self.device)

    def graph(self) -> Graph:
        h = C.c_void_p()
        check(_L().dg_graph_create_from_device_edges(self._h, C.byref(h)))
        return Graph(self.v_num, handle=h, device=self.device)

    def close(self):
        if getattr(self, "_h", None):
            _L().dg_edges_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def common_neighbours(src, dst, v_num: int, undirected: bool = True, device: int = 0) -> np.ndarray:
    """Common-neighbour count of every edge (the reference's gcn tool, src/tools/gcn.cpp),
    computed on the device by dg_common_neighbours; int32 in input order."""
    s = np.ascontiguousarray(src, dtype=np.uint32)
    d = np.ascontiguousarray(dst, dtype=np.uint32)
    out = np.empty(s.size, np.int32)
    check(lib().dg_common_neighbours(s.ctypes.data if s.size else None, d.ctypes.data if d.size else None, s.size,
                                     v_num, int(undirected), device, out.ctypes.data if s.size else None))
    return out
