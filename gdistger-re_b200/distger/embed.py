"""The whole embedding job in one call: walk rounds streamed into SGNS.

Same loop as the C++ host program (host/huge_walk.cpp), over the same C ABI:
round 1 with walker_num x init_round walkers, then walker_num walkers a round,
30 rounds (walk.hpp:609-782); each round's walks are trained where they lie in
HBM (dg_pipeline_round) with the round's learning rate from the schedule
(word2vec.cu:1279-1290: ExponentialDecayLR(alpha, 0.1), one get_lr() per round).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from ._lib import check, lib
from .sgns import SGNS, CosineAnnealingLR, CustomLR, ExponentialDecayLR, FixedLR, StepDecayLR
from .walk import LAST_ROUND, Graph


def make_lr(kind: str, alpha: float, rounds: int):
    if kind == "exp":
        return ExponentialDecayLR(alpha, 0.1)
    if kind == "fixed":
        return FixedLR(alpha)
    if kind == "cosine":
        return CosineAnnealingLR(alpha, alpha * 1e-4, rounds)
    if kind == "step":
        return StepDecayLR(alpha, 0.5, 3)
    if kind == "custom":
        return CustomLR(alpha)
    raise ValueError("lr must be exp, fixed, cosine, step or custom")


def embed(graph: Graph, walker_num: int | None = None, mode: str = "plain", size: int = 128, window: int = 10,
          negative: int = 5, batch_size: int = 21, sample: float = 1e-3, alpha: float = 0.01, iter: int = 1,
          min_count: int = 0, rounds: int = LAST_ROUND, init_round: int = 5, min_len: int = 20, lr: str = "exp",
          train_from: int = 1, seed: int = 1, master_rows: int = 0, workers: int = 0, deterministic: int = 0,
          max_len: int = 64, keep_trainer: bool = False, device: int = 0, plain_shape: int | None = None) -> dict:
    """Runs the job on `graph` and returns the embedding in vertex order plus the job's counters.
    deterministic = 2 trains by adjoint gradient steps (see dg_sgns_params); plain_shape
    selects a launch shape of the plain kernel (SGNS.set_shape)."""
    t0 = time.perf_counter()
    v_num = graph.v_num
    walker_num = walker_num or v_num
    out_deg, in_deg = graph.degrees()
    counts = out_deg + in_deg   # huge_walk.cpp:40-44
    sgns = SGNS(v_num, counts, size=size, window=window, negative=negative, batch_size=batch_size, sample=sample,
                alpha=alpha, iter=iter, min_count=min_count, mode=mode, seed=seed, master_rows=master_rows,
                workers=workers, deterministic=deterministic, device=device)
    if plain_shape is not None:
        sgns.set_shape(plain_shape)
    wp = _lib.WalkParams(min_len=min_len, init_round=init_round, walker_num=walker_num, max_len=max_len, seed=seed)
    sched = make_lr(lr, alpha, rounds)
    L = lib()
    acc = dict(walk_ms=0.0, train_ms=0.0, device_ms=0.0, steps=0, footprints=0, draws=0, words=0, pairs=0)
    per_round = []
    t1 = time.perf_counter()
    for r in range(1, rounds + 1):
        if r >= train_from:
            a = sched.get_lr()
            info = _lib.PipelineInfo()
            check(L.dg_pipeline_round(graph.handle, sgns.handle, C.byref(wp), r, 0, C.c_float(a), C.byref(info), None))
            w, t = info.walk, info.train
            acc["train_ms"] += t.train_ms
            acc["device_ms"] += info.total_ms
            acc["words"] += t.words
            acc["pairs"] += t.pairs
        else:
            a = None
            ph = C.c_void_p()
            check(L.dg_walk_run_round(graph.handle, C.byref(wp), r, 0, C.byref(ph)))
            w = _lib.RoundInfo()
            check(L.dg_paths_get_info(ph, C.byref(w)))
            L.dg_paths_free(ph)
            acc["device_ms"] += w.walk_ms
        acc["walk_ms"] += w.walk_ms
        acc["steps"] += w.steps
        acc["footprints"] += w.footprints
        acc["draws"] += w.draws
        per_round.append({"round": r, "walks": w.n_walks, "steps": w.steps, "delta_h": abs(w.delta_h), "alpha": a})
    t2 = time.perf_counter()
    acc["workers"] = sgns.workers
    if keep_trainer:
        acc["trainer"] = sgns
    else:
        rows, ids = sgns.embedding()
        emb = np.zeros((v_num, size), np.float32)
        emb[ids] = rows
        acc["embedding"] = emb
        sgns.close()
    acc.update(rounds=per_round, rounds_wall_s=t2 - t1, wall_s=t2 - t0,
               walk_steps_per_s=acc["steps"] / (acc["walk_ms"] * 1e-3) if acc["walk_ms"] else 0.0,
               words_per_s=acc["words"] / (acc["train_ms"] * 1e-3) if acc["train_ms"] else 0.0)
    return acc
