"""bench.py's multi-process path on CPU: two ranks over gloo reduce the timed
quantities as the bench does (time: max over ranks; work: sum over ranks), and
the reference arm runs on rank 0 only (other ranks return without work)."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, q):
    os.environ.update(WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    r, world, local, pg = bench.dist_init()
    try:
        t = bench.reduce_max(pg, 1.5 + r)          # per-rank device seconds
        w = bench.reduce_sum(pg, 1000.0 * (r + 1))  # per-rank footprints
        bench.barrier(pg)
        q.put((r, world, t, w))
    finally:
        pg.destroy_process_group()


def test_two_ranks_reduce_like_the_bench():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 2, 2.5, 3000.0), (1, 2, 2.5, 3000.0)]


def test_reference_arm_runs_on_rank0_only(capsys):
    sys.path.insert(0, ROOT)
    import bench
    assert bench.run_reference(None, 1, 2, None) is None   # rank 1: no work, no output
    assert capsys.readouterr().out == ""
