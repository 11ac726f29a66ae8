"""Host-side mirror of the reference's walk interface over the CUDA library.

`WalkEngine` keeps the names and argument meaning of the reference's
WalkEngine<real_t, uint32_t> (include/walk.hpp:389-1044): set_init_round /
set_minLength ignore 0 (walk.hpp:488-496), load_graph(v_num, graph_path,
partition_path, make_undirected) (graph.hpp:642), random_walk(...) runs the
round loop of internal_random_walk (walk.hpp:609-782): round 1 with
walker_num * init_round walkers, then walker_num walkers per round, one walk file
`<prefix>-0-<round>.txt` per round, relative entropy after each round, stop after
round 30 (walk.hpp:740).  All walking happens in the CUDA kernel.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, lib

EDGE_DTYPE = np.dtype([("src", "<u4"), ("dst", "<u4"), ("data", "<f4")])
LAST_ROUND = 30  # walk.hpp:740


class Graph:
    """Device CSR (GraphEngine::load_graph, graph.hpp:642-824)."""

    def __init__(self, v_num: int, graph_path: str | None = None, edges: np.ndarray | None = None,
                 make_undirected: bool = False, device: int = 0, handle=None):
        h = C.c_void_p()
        if handle is not None:
            h = handle
        elif edges is not None:
            edges = np.ascontiguousarray(edges, dtype=EDGE_DTYPE)
            check(lib().dg_graph_create_from_edges(edges.ctypes.data if edges.size else None, edges.size,
                                                   v_num, int(make_undirected), device, C.byref(h)))
        elif graph_path is not None:
            check(lib().dg_graph_create(graph_path.encode(), v_num, int(make_undirected), device, C.byref(h)))
        else:
            raise ValueError("need graph_path or edges")
        self._h = h
        self.device = device
        info = _lib.GraphInfo()
        check(lib().dg_graph_get_info(h, C.byref(info)))
        self.v_num = info.v_num
        self.m = info.m
        self.device_bytes = info.device_bytes
        self.threshold_ms = info.threshold_ms

    @property
    def handle(self):
        return self._h

    def csr(self) -> dict:
        off = np.empty(self.v_num + 1, np.uint64)
        nbr = np.empty(self.m, np.uint32)
        thr = np.empty(self.m, np.uint32)
        od = np.empty(self.v_num, np.uint32)
        idg = np.empty(self.v_num, np.uint32)
        check(lib().dg_graph_copy_csr(self._h, off.ctypes.data, nbr.ctypes.data if self.m else None,
                                      thr.ctypes.data if self.m else None, od.ctypes.data, idg.ctypes.data))
        return {"offsets": off, "nbr": nbr, "thresholds": thr, "out_deg": od, "in_deg": idg}

    def degrees(self):
        """(out_degree, in_degree) without copying the CSR itself."""
        od = np.empty(self.v_num, np.uint32)
        idg = np.empty(self.v_num, np.uint32)
        check(lib().dg_graph_copy_csr(self._h, None, None, None, od.ctypes.data, idg.ctypes.data))
        return od, idg

    def visits(self) -> np.ndarray:
        f = np.empty(self.v_num, np.uint32)
        check(lib().dg_graph_copy_visits(self._h, f.ctypes.data))
        return f

    def close(self):
        if getattr(self, "_h", None):
            lib().dg_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Paths:
    """One round of walks, resident on the device."""

    def __init__(self, handle, graph: Graph):
        self._h = handle
        self._graph = graph  # keeps the graph (and its stream) alive
        info = _lib.RoundInfo()
        check(lib().dg_paths_get_info(handle, C.byref(info)))
        self.info = info

    @property
    def handle(self):
        return self._h

    def to_numpy(self):
        n = self.info.n_walks
        offs = np.empty(n + 1, np.uint64)
        verts = np.empty(self.info.footprints, np.uint32)
        check(lib().dg_paths_copy(self._h, offs.ctypes.data, verts.ctypes.data if verts.size else None))
        return offs, verts

    def write_text(self, path: str) -> None:
        check(lib().dg_paths_write_text(self._h, path.encode()))

    def close(self):
        if getattr(self, "_h", None):
            lib().dg_paths_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class RoundResult:
    round: int
    n_walks: int
    steps: int
    footprints: int
    walk_ms: float
    relative_entropy: float
    delta_h: float
    output_path: str | None


class WalkEngine:
    """Mirror of WalkEngine<real_t, uint32_t>: the HuGE-style information-oriented walk."""

    def __init__(self, device: int = 0, seed: int = 0, max_len: int = 64):
        self.device = device
        self.seed = seed
        self.max_len = max_len
        self.init_round = 5   # walk.hpp:405
        self.minLength = 20   # walk.hpp:404
        self.graph: Graph | None = None

    def set_init_round(self, init_round: int) -> None:
        if init_round != 0:
            self.init_round = init_round

    def set_minLength(self, min_length: int) -> None:
        if min_length != 0:
            self.minLength = min_length

    def load_graph(self, v_num: int, graph_path: str, partition_path: str = "", make_undirected: bool = False,
                   edges: np.ndarray | None = None) -> None:
        if partition_path:
            raise ValueError("partition files select an MPI partition; one GPU holds the whole graph")
        self.graph = Graph(v_num, graph_path=None if edges is not None else graph_path, edges=edges,
                           make_undirected=make_undirected, device=self.device)

    def get_vertex_num(self) -> int:
        return self.graph.v_num

    def params(self, walker_num: int) -> _lib.WalkParams:
        return _lib.WalkParams(min_len=self.minLength, init_round=self.init_round, walker_num=walker_num,
                               max_len=self.max_len, seed=self.seed)

    def autotune(self, walker_num: int, round_index: int = 2, n_walkers: int = 0) -> dict:
        """Times the walk kernel's launch shapes on this graph and keeps the fastest
        (walks are identical under every shape; visit counts are rolled back)."""
        if self.graph is None:
            raise RuntimeError("load_graph first")
        info = _lib.TuneInfo()
        check(lib().dg_walk_autotune(self.graph.handle, C.byref(self.params(walker_num)), round_index, n_walkers,
                                     C.byref(info)))
        return info.as_dict()

    def run_round(self, walker_num: int, round_index: int, n_walkers: int = 0) -> Paths:
        if self.graph is None:
            raise RuntimeError("load_graph first")
        p = self.params(walker_num)
        h = C.c_void_p()
        check(lib().dg_walk_run_round(self.graph.handle, C.byref(p), round_index, n_walkers, C.byref(h)))
        return Paths(h, self.graph)

    def random_walk(self, walker_num: int, output_path_prefix: str | None = None, consumer=None,
                    last_round: int = LAST_ROUND, verbose: bool = False) -> list:
        """Round loop of internal_random_walk (walk.hpp:609-782), rank 0 of 1."""
        results = []
        for r in range(1, last_round + 1):
            paths = self.run_round(walker_num, r)
            out = None
            if output_path_prefix:
                out = f"{output_path_prefix}-0-{r}.txt"
                paths.write_text(out)
            i = paths.info
            results.append(RoundResult(r, i.n_walks, i.steps, i.footprints, i.walk_ms, i.relative_entropy,
                                       i.delta_h, out))
            if verbose:
                print(f"round {r}: walks {i.n_walks} steps {i.steps} Delat RE {abs(i.delta_h):g}")
            if consumer is not None:
                consumer(r, paths)
            paths.close()
        return results
