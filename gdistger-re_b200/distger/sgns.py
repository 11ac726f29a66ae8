"""Host-side mirror of the reference's SGNS trainers over the CUDA library.

`SGNS` carries the trainer flags of word2vec.cu (train_corpus_cuda,
word2vec.cu:1545-1565) and dsgl (dsgl.hpp:1497-1548): size, window, negative,
batch_size, sample, alpha, iter, min_count.  mode="plain" follows word2vec.cu's
skip_gram_kernel update rule on FP32 rows; mode="minibatch" follows dsgl's
shared-negative minibatches on BF16 rows; mode="cbow" follows cbow_kernel (the
reference's default, -cbow 1) and mode="sg_shared" __sgNegReuse (-cbow 0
-reuse-neg 1: one negative set per walk, full window), both on FP32 rows.  The learning-rate schedules of
include/lr_scheduler.hpp are restated below for the per-round loop.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check, lib

MODES = {"plain": 0, "minibatch": 1, "plain_bf16": 2, "cbow": 3, "sg_shared": 4, "cbow_bf16": 5}


class SGNS:
    def __init__(self, v_num: int, vertex_counts: np.ndarray, size: int = 128, window: int = 5, negative: int = 5,
                 batch_size: int = 11, sample: float = 1e-3, alpha: float = 0.025, iter: int = 1,
                 min_count: int = 5, mode: str = "plain", deterministic: bool = False, seed: int = 1,
                 table_size: int = 0, master_rows: int = 0, workers: int = 0, device: int = 0, hs: bool = False):
        counts = np.ascontiguousarray(vertex_counts, dtype=np.uint32)
        if counts.size != v_num:
            raise ValueError("vertex_counts must have v_num entries")
        p = _lib.SgnsParams(size=size, window=window, negative=negative, batch_size=batch_size, sample=sample,
                            alpha=alpha, iter=iter, min_count=min_count, mode=MODES[mode],
                            deterministic=int(deterministic), seed=seed, table_size=table_size,
                            master_rows=master_rows, workers=workers, hs=int(hs))
        h = C.c_void_p()
        check(lib().dg_sgns_create(C.byref(p), v_num, counts.ctypes.data, device, C.byref(h)))
        self._h = h
        self.params = p
        self.v_num = v_num
        self.size = size
        self.mode = mode
        info = _lib.SgnsInfo()
        check(lib().dg_sgns_get_info(h, C.byref(info)))
        self.vocab_size = info.vocab_size
        self.master_rows = info.master_rows
        self.workers = info.workers
        self.bf_staged = bool(info.bf_staged)
        self.train_words = info.train_words
        self.table_size = info.table_size

    @property
    def handle(self):
        return self._h

    def autotune(self, paths) -> dict:
        """Times the plain kernel's launch shapes on these walks and keeps the fastest
        (rows and pass counter restored)."""
        info = _lib.TuneInfo()
        check(lib().dg_sgns_autotune(self._h, paths.handle, C.byref(info)))
        return info.as_dict()

    def set_shape(self, shape: int) -> None:
        """Selects launch shape `shape` of the plain kernel (an index of the list
        autotune times)."""
        check(lib().dg_sgns_set_shape(self._h, int(shape)))

    def train_paths(self, paths, alpha: float = 0.0) -> _lib.TrainInfo:
        info = _lib.TrainInfo()
        check(lib().dg_sgns_train_paths(self._h, paths.handle, alpha, C.byref(info)))
        return info

    def train_host(self, offsets: np.ndarray, verts: np.ndarray, alpha: float = 0.0) -> _lib.TrainInfo:
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        verts = np.ascontiguousarray(verts, dtype=np.uint32)
        info = _lib.TrainInfo()
        check(lib().dg_sgns_train_host(self._h, offsets.ctypes.data, offsets.size - 1,
                                       verts.ctypes.data if verts.size else None, alpha, C.byref(info)))
        return info

    def embedding(self):
        rows = np.empty((self.vocab_size, self.size), np.float32)
        ids = np.empty(self.vocab_size, np.uint32)
        n = C.c_uint32()
        check(lib().dg_sgns_copy_embedding(self._h, rows.ctypes.data, ids.ctypes.data, C.byref(n)))
        return rows, ids

    def output_rows(self) -> np.ndarray:
        rows = np.empty((self.vocab_size, self.size), np.float32)
        check(lib().dg_sgns_copy_output(self._h, rows.ctypes.data))
        return rows

    def set_rows(self, input_rows=None, output_rows=None) -> None:
        a = None if input_rows is None else np.ascontiguousarray(input_rows, dtype=np.float32)
        b = None if output_rows is None else np.ascontiguousarray(output_rows, dtype=np.float32)
        check(lib().dg_sgns_set_rows(self._h, None if a is None else a.ctypes.data,
                                     None if b is None else b.ctypes.data))

    def tables(self):
        table = np.empty(self.table_size, np.int32)
        keep = np.empty(self.vocab_size, np.uint32)
        v2w = np.empty(self.v_num, np.int32)
        et = np.empty(1001, np.float32)
        check(lib().dg_sgns_copy_tables(self._h, table.ctypes.data, keep.ctypes.data, v2w.ctypes.data,
                                        et.ctypes.data))
        return {"table": table, "keep_thr": keep, "v2w": v2w, "exp_table": et}

    @staticmethod
    def _pairs(inputs, outputs, negatives, batch: int, negative: int):
        inp = np.ascontiguousarray(inputs, dtype=np.uint32)
        outp = np.ascontiguousarray(outputs, dtype=np.uint32)
        neg = np.ascontiguousarray(negatives, dtype=np.uint32)
        if inp.size != outp.size:
            raise ValueError("inputs and outputs differ in length")
        p = _lib.SgnsPairs(inputs=inp.ctypes.data if inp.size else None,
                           outputs=outp.ctypes.data if outp.size else None,
                           negatives=neg.ctypes.data if neg.size else None, n_pairs=inp.size, batch=batch,
                           negative=negative)
        return p, (inp, outp, neg)

    def loss_grad(self, inputs, outputs, negatives, batch: int = 21, negative: int = 5, grad: bool = True):
        """SGNS loss over explicit minibatches at the current rows and its gradient
        (hand-written backward kernel, deterministic): (loss, grad_in, grad_out)."""
        p, keep = self._pairs(inputs, outputs, negatives, batch, negative)
        loss = C.c_double()
        gi = np.empty((self.vocab_size, self.size), np.float32) if grad else None
        go = np.empty((self.vocab_size, self.size), np.float32) if grad else None
        check(lib().dg_sgns_loss_grad(self._h, C.byref(p), C.byref(loss), gi.ctypes.data if grad else None,
                                      go.ctypes.data if grad else None))
        return loss.value, gi, go

    def adjoint_step(self, inputs, outputs, negatives, alpha: float, batch: int = 21, negative: int = 5) -> float:
        """Deterministic step rows -= alpha * gradient; returns the loss before the step."""
        p, keep = self._pairs(inputs, outputs, negatives, batch, negative)
        loss = C.c_double()
        check(lib().dg_sgns_adjoint_step(self._h, C.byref(p), C.c_float(alpha), C.byref(loss)))
        return loss.value

    def write_embedding(self, path: str) -> None:
        check(lib().dg_sgns_write_embedding(self._h, path.encode()))

    def close(self):
        if getattr(self, "_h", None):
            lib().dg_sgns_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------- include/lr_scheduler.hpp ----
class LR:
    def __init__(self, initial_lr: float):
        self.initial_lr = initial_lr
        self.step = 0


class FixedLR(LR):
    def get_lr(self) -> float:
        return self.initial_lr


class ExponentialDecayLR(LR):
    """initial_lr * exp(-decay_rate * step), step post-incremented (lr_scheduler.hpp:23-31)."""

    def __init__(self, initial_lr: float, decay_rate: float):
        super().__init__(initial_lr)
        self.decay_rate = decay_rate

    def get_lr(self) -> float:
        lr = float(np.float32(self.initial_lr) * np.float32(math.exp(-np.float32(self.decay_rate) * self.step)))
        self.step += 1
        return lr


class CosineAnnealingLR(LR):
    def __init__(self, initial_lr: float, min_lr: float, t_max: int):
        super().__init__(initial_lr)
        self.min_lr = min_lr
        self.t_max = t_max

    def get_lr(self) -> float:
        cosine = math.cos(math.pi * self.step / self.t_max)
        lr = self.min_lr + 0.5 * (self.initial_lr - self.min_lr) * (1 + cosine)
        self.step += 1
        return lr


class StepDecayLR(LR):
    def __init__(self, initial_lr: float, decay_factor: float, step_size: int):
        super().__init__(initial_lr)
        self.decay_factor = decay_factor
        self.step_size = step_size

    def get_lr(self) -> float:
        factor = self.step // self.step_size
        self.step += 1
        return self.initial_lr * self.decay_factor ** factor


class CustomLR(LR):
    def get_lr(self) -> float:
        if self.step % 5 == 0:
            self.initial_lr *= 0.8
        self.step += 1
        return self.initial_lr
