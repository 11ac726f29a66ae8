"""The allocation-free minibatch trainer against the handle-based one.

dg_sgns_minibatch_train_noalloc exists for callers that cannot allocate device
memory (a framework whose memory pool owns the device memory, a latency-bound
loop that cannot pay cudaMalloc's device synchronisation): the caller owns every
buffer and the trainer's scratch lives in a fixed array inside the library.
Here the caller's buffers come from torch, are filled with the tables and
initial rows of a handle-based trainer with the same parameters, and two calls
in a row must leave the rows equal to what the handle's two dg_sgns_train_host
calls produce (deterministic mode: identical, so the tolerance of the other SGNS
tests, exact FP32 agreement, applies).  Hogwild runs (several workers racing)
must report the handle path's counters and stay within the relative Frobenius
distance the other Hogwild tests allow.

The file sorts last so that, in a run that stops at the first failure, every
other GPU test has run before it.  It does not depend on running last: each
call clears the library's counters, and every test builds its own buffers and
its own handle trainer.
"""
import ctypes as C
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
pytestmark = pytest.mark.gpu


def _walks_and_counts():
    import dgoracle
    from distger import graphgen
    rounds, _, _ = dgoracle.load_golden(os.path.join(GOLDEN, "tiny200_ref_walks.npz"))
    edges = graphgen.read_edges(os.path.join(GOLDEN, "tiny200.bin"))
    csr = dgoracle.Csr(edges, 200, undirected=True)
    return rounds[0], (csr.out_deg + csr.in_deg).astype(np.uint32)


def _rows_from_device(bf16_t, master_t, n_master):
    bits = bf16_t.cpu().numpy().astype(np.uint16).astype(np.uint32) << 16
    rows = bits.view(np.float32).copy()
    rows[:n_master] = master_t.cpu().numpy()[:n_master]
    return rows


def test_noalloc_minibatch_matches_handle_two_calls(distger_lib):
    import torch
    from distger import _lib
    from distger._lib import check, lib
    from distger.sgns import SGNS

    (offs, verts), counts = _walks_and_counts()
    size, n_master = 64, 16
    ref = SGNS(200, counts, size=size, window=5, negative=5, sample=1e-3, alpha=0.025, min_count=0,
               mode="minibatch", deterministic=True, seed=11, table_size=1_000_000, master_rows=n_master)
    t = ref.tables()
    rows0, _ = ref.embedding()
    vs = ref.vocab_size
    dev = torch.device("cuda:0")
    u16 = (rows0.view(np.uint32) >> 16).astype(np.uint16)
    in_bf = torch.from_numpy(u16.view(np.int16).copy()).to(dev)
    out_bf = torch.zeros((vs, size), dtype=torch.int16, device=dev)
    in_m = torch.from_numpy(rows0[:n_master].copy()).to(dev)
    out_m = torch.zeros((n_master, size), dtype=torch.float32, device=dev)
    v2w = torch.from_numpy(t["v2w"]).to(dev)
    keep = torch.from_numpy(t["keep_thr"].view(np.int32)).to(dev)
    table = torch.from_numpy(t["table"]).to(dev)
    expt = torch.from_numpy(t["exp_table"]).to(dev)
    torch.cuda.synchronize()

    for call in range(2):
        lo, hi = 50 * call, 50 * call + 50
        o = (offs[lo:hi + 1] - offs[lo]).astype(np.uint64)
        v = verts[int(offs[lo]):int(offs[hi])].astype(np.uint32)
        want = ref.train_host(o, v)
        d_off = torch.from_numpy(o.view(np.int64)).to(dev)
        d_v = torch.from_numpy(v.view(np.int32)).to(dev)
        torch.cuda.synchronize()
        a = _lib.MinibatchArgs(verts=d_v.data_ptr(), offsets=d_off.data_ptr(), n_walks=hi - lo,
                               v2w=v2w.data_ptr(), keep_thr=keep.data_ptr(), table=table.data_ptr(),
                               table_size=table.numel(), exp_table=expt.data_ptr(), vocab_size=vs,
                               in_bf16=in_bf.data_ptr(), out_bf16=out_bf.data_ptr(), in_master=in_m.data_ptr(),
                               out_master=out_m.data_ptr(), n_master=n_master, size=size, window=5, negative=5,
                               alpha=0.025, seed=11, pass_=call, deterministic=1)
        got = _lib.TrainInfo()
        check(lib().dg_sgns_minibatch_train_noalloc(C.byref(a), None, C.byref(got)))
        assert (got.words, got.trained, got.pairs) == (want.words, want.trained, want.pairs)
        exp_in, _ = ref.embedding()
        exp_out = ref.output_rows()
        np.testing.assert_array_equal(_rows_from_device(in_bf, in_m, n_master), exp_in, err_msg=f"call {call}")
        np.testing.assert_array_equal(_rows_from_device(out_bf, out_m, n_master), exp_out, err_msg=f"call {call}")


def _device_state(ref, size, n_master, dev):
    import torch
    t = ref.tables()
    rows0, _ = ref.embedding()
    vs = ref.vocab_size
    u16 = (rows0.view(np.uint32) >> 16).astype(np.uint16)
    st = dict(in_bf=torch.from_numpy(u16.view(np.int16).copy()).to(dev),
              out_bf=torch.zeros((vs, size), dtype=torch.int16, device=dev),
              in_m=torch.from_numpy(rows0[:n_master].copy()).to(dev),
              out_m=torch.zeros((max(n_master, 1), size), dtype=torch.float32, device=dev),
              v2w=torch.from_numpy(t["v2w"]).to(dev), keep=torch.from_numpy(t["keep_thr"].view(np.int32)).to(dev),
              table=torch.from_numpy(t["table"]).to(dev), expt=torch.from_numpy(t["exp_table"]).to(dev))
    torch.cuda.synchronize()
    return st


@pytest.fixture(scope="module")
def walks10k():
    import distger
    from distger import graphgen
    edges = graphgen.chung_lu(10_000, 100_000, 2.2, seed=0)
    eng = distger.WalkEngine(seed=5)
    eng.load_graph(10_000, "", make_undirected=True, edges=edges)
    p = eng.run_round(10_000, 1, n_walkers=4000)
    offs, verts = p.to_numpy()
    od, idg = eng.graph.degrees()
    p.close()
    eng.graph.close()
    return offs, verts, (od + idg).astype(np.uint32)


def _rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b.astype(np.float64)))


@pytest.mark.parametrize("size,negative,workers", [(64, 5, 8), (256, 14, 0)],
                         ids=["8-workers", "array-bound-workers"])
def test_noalloc_hogwild_matches_handle(distger_lib, walks10k, size, negative, workers):
    """Several workers racing on a 10,000-vertex power-law graph: the same counters
    as the handle path with the same worker count (walks are sliced per worker),
    and rows no further from a handle run than 3x the distance between two handle
    runs plus 1e-3 (Hogwild runs differ from each other by their races).  size 256
    with 14 negatives needs about 1 MB of scratch per worker, so the 16 MiB array
    admits 17 workers, fewer than the default of 128: the handle path runs with
    that count."""
    import torch
    from distger import _lib
    from distger._lib import check, lib
    from distger.sgns import SGNS

    offs, verts, counts = walks10k
    n_master = 256
    per_worker = (32 * negative * size * 2 + 64 * size) * 4
    eff = min(workers or 128, (16 << 20) // per_worker)
    kw = dict(size=size, window=5, negative=negative, sample=1e-3, alpha=0.025, min_count=0, mode="minibatch",
              seed=5, table_size=1_000_000, master_rows=n_master)
    runs = []
    for _ in range(2):
        ref = SGNS(counts.size, counts, deterministic=False, workers=eff, **kw)
        want = ref.train_host(offs, verts)
        runs.append((want, ref.embedding()[0], ref.output_rows()))
        ref.close()
    noise = max(_rel(runs[0][1], runs[1][1]), _rel(runs[0][2], runs[1][2]))
    ref = SGNS(counts.size, counts, deterministic=False, workers=eff, **kw)
    dev = torch.device("cuda:0")
    st = _device_state(ref, size, n_master, dev)
    ref.close()
    d_off = torch.from_numpy(offs.astype(np.uint64).view(np.int64)).to(dev)
    d_v = torch.from_numpy(verts.astype(np.uint32).view(np.int32)).to(dev)
    torch.cuda.synchronize()
    a = _lib.MinibatchArgs(verts=d_v.data_ptr(), offsets=d_off.data_ptr(), n_walks=offs.size - 1,
                           v2w=st["v2w"].data_ptr(), keep_thr=st["keep"].data_ptr(), table=st["table"].data_ptr(),
                           table_size=st["table"].numel(), exp_table=st["expt"].data_ptr(),
                           vocab_size=runs[0][1].shape[0], in_bf16=st["in_bf"].data_ptr(),
                           out_bf16=st["out_bf"].data_ptr(), in_master=st["in_m"].data_ptr(),
                           out_master=st["out_m"].data_ptr(), n_master=n_master, size=size, window=5,
                           negative=negative, alpha=0.025, seed=5, pass_=0, deterministic=0, workers=workers)
    got = _lib.TrainInfo()
    check(lib().dg_sgns_minibatch_train_noalloc(C.byref(a), None, C.byref(got)))
    want = runs[0][0]
    assert (got.words, got.trained, got.pairs, got.rows) == (want.words, want.trained, want.pairs, want.rows)
    mine_in = _rows_from_device(st["in_bf"], st["in_m"], n_master)
    mine_out = _rows_from_device(st["out_bf"], st["out_m"], n_master)
    assert np.isfinite(mine_in).all() and np.isfinite(mine_out).all()
    d = max(_rel(mine_in, runs[0][1]), _rel(mine_out, runs[0][2]))
    print(f"noalloc vs handle {d:.3e}, handle vs handle {noise:.3e}")
    assert d <= 3 * noise + 1e-3


def test_noalloc_rejects_unsupported_size(distger_lib):
    from distger import DistgerError, _lib
    from distger._lib import check, lib
    a = _lib.MinibatchArgs(verts=1, offsets=1, n_walks=1, v2w=1, keep_thr=1, table=1, table_size=1, exp_table=1,
                           vocab_size=1, in_bf16=1, out_bf16=1, in_master=1, out_master=1, n_master=1, size=512,
                           window=5, negative=5, alpha=0.025, seed=1, pass_=0, deterministic=1)
    with pytest.raises(DistgerError) as e:
        check(lib().dg_sgns_minibatch_train_noalloc(C.byref(a), None, None))
    assert e.value.code == -1 and "size 512" in str(e.value)
