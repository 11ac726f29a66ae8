"""Exact replay of the benched staged-rows kernel (sgns_plain_pipe_kernel).

Run by one warp (launch shape 12: 32 threads, 2 staged pairs; one worker), the
kernel's result is fixed by program order, so the CPU model oracle/dg_oracle_pipe.c
(rows of pair m copied after the updates of pairs < m - 1, context rows of the
last two pairs taken from their updated copies, the centre's output row in
registers, FP32 rows and masters updated by additions) must match it bit for bit:
  * FP32 rows (the plain form's default shape is this kernel with two warps per
    block);
  * BF16 rows with FP32 masters (the bench's headline form): a BF16 row is
    overwritten with the warp's stochastically rounded copy; the kernel rounds
    with the cvt.rs.bf16x2.f32 convert, the model with the software rule (16 noise
    bits added below the kept mantissa, then truncation), so equality also pins
    the convert to that rule.
Two passes in a row, so that the second starts from rows the first wrote.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ONE_WARP_STAGED = 12


@pytest.fixture(scope="module")
def big_round():
    import distger
    from distger import graphgen
    edges = graphgen.chung_lu(200_000, 2_000_000, 2.2, seed=1)
    eng = distger.WalkEngine(seed=5)
    eng.load_graph(200_000, "", make_undirected=True, edges=edges)
    p = eng.run_round(200_000, 1, n_walkers=600)
    od, idg = eng.graph.degrees()
    yield p, od + idg
    p.close()


@pytest.mark.parametrize("mode,size,negative,window", [("plain", 128, 5, 10), ("plain", 64, 3, 5),
                                                       ("plain_bf16", 128, 5, 10), ("plain_bf16", 128, 7, 4)])
def test_one_warp_staged_bit_exact(distger_lib, oracle, big_round, mode, size, negative, window):
    from distger.sgns import SGNS
    p, counts = big_round
    s = SGNS(counts.size, counts, size=size, window=window, negative=negative, sample=1e-3, alpha=0.025,
             min_count=0, seed=3, table_size=1_000_000, mode=mode, workers=1)
    bf16 = mode == "plain_bf16"
    if bf16:
        assert s.bf_staged and 0 < s.master_rows < counts.size
    s.set_shape(ONE_WARP_STAGED)
    rows_in = np.ascontiguousarray(s.embedding()[0])
    rows_out = np.ascontiguousarray(s.output_rows())
    t = s.tables()
    offs, verts = p.to_numpy()
    for it in range(2):
        info = s.train_paths(p)
        st = oracle.sgns_pipe(t, rows_in, rows_out, offs, verts, size, window, negative, 0.025, 3, it, stages=2,
                              bf16=bf16, n_master=s.master_rows if bf16 else 0)
        assert (info.words, info.trained, info.pairs) == (st.words, st.trained, st.pairs)
        got_in, _ = s.embedding()
        got_out = s.output_rows()
        assert np.array_equal(got_in.view(np.uint32), rows_in.view(np.uint32)), f"pass {it}"
        assert np.array_equal(got_out.view(np.uint32), rows_out.view(np.uint32)), f"pass {it}"
    s.close()
