#!/usr/bin/env python
"""Benchmark of DistGER's embedding hot path on B200: walk rounds streamed into SGNS.

Workload (N=1, the default): the Twitter-shaped graph -- Chung-Lu power law,
exponent 1.9, 41,652,230 vertices, 2.417e9 edge draws leaving ~1.47e9 unique
undirected edges, expected degrees capped at 3M, unweighted, generated and built
into the CSR on the device -- with the reference walk defaults (--min_L 20,
--min_R 5, w = V walkers per round, walks of at most 32 footprints) and SGNS
d=128, window 10, negative 5, sample 1e-3, alpha 0.01, iter 1; headline form:
the plain rule on BF16 rows with FP32 masters, FP32 plain measured beside it.
--bench-workload c2_youtube (1,138,499 vertices, exponent 2.1, ~2.99M edges,
FP32 plain) and c3_livejournal (2,238,731 vertices, exponent 2.3, 14M edge
draws, BF16 against FP32) are the smaller lines.  One step = one walk round of
V walks + SGNS over those walks.  Synthetic data: none of the paper's graphs
ship with the reference.

value  = walk-steps embedded per second: footprints walked and trained per
         second of device time (CUDA events from the walk launch to the end of
         training), summed over ranks / max over ranks of the time;
e2e    = the same through the C ABI with host buffers: walks copied to pinned
         host memory (dg_paths_copy) and trained from there (dg_sgns_train_host),
         copies inside the timed region;
--impl reference: the reference's own walk engine + dsgl trainer compiled from
         its sources (oracle/_ref/ref_embed) on the host cores, same metric.

Multi-GPU: the path does not shard (one process, one GPU per the task); N GPUs
run N independent replicas (weak scaling), each rank on LOCAL_RANK's device.
"""
from __future__ import annotations

import argparse
import csv
import ctypes as C
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gdistger-re_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "walk-steps/s + SGNS words/s, end-to-end embed time; BF16 vs FP32 plain at equal AUC"
UNIT = "walk-steps/s"
BF16_FORMS = ("plain_bf16", "minibatch", "cbow_bf16")   # trainer forms with BF16 rows and FP32 masters
SGNS_HP = {"size": 128, "window": 10, "negative": 5, "sample": 1e-3, "alpha": 0.01, "iter": 1, "min_count": 0}
# Bench workloads.  c5_twitter (the default): the Twitter-shaped graph, 41,652,230
# vertices, Chung-Lu exponent 1.9, expected degrees capped at 3M, 2.417e9 edge draws
# leaving ~1.47e9 unique undirected edges, unweighted; --min_R 5 (run.sh:45), walks
# of at most 32 footprints; headline form: BF16 rows with FP32 masters (the plain
# rule), FP32 plain beside it.  c2_youtube: the YouTube-shaped graph, FP32 plain.
# c3_livejournal: the LiveJournal-shaped graph (2,238,731 vertices, exponent 2.3,
# 14M undirected edge draws, weighted), BF16 rows against FP32 plain.
BENCH = {
    "c5_twitter": dict(graph="twitter-shaped chung-lu, generated on the device", source="device",
                       vertices=41_652_230, draws=2_417_000_000, exponent=1.9, max_degree=3_000_000, weighted=False,
                       min_L=20, min_R=5, max_len=32, headline="plain_bf16", **SGNS_HP),
    "c2_youtube": dict(graph="youtube-shaped chung-lu", source="host", vertices=1_138_499,
                       undirected_edges=2_990_443, exponent=2.1, max_degree=28_000, weighted=True,
                       min_L=20, min_R=10, max_len=64, headline="plain", **SGNS_HP),
    "c3_livejournal": dict(graph="livejournal-shaped chung-lu", source="host", vertices=2_238_731,
                           undirected_edges=14_000_000, exponent=2.3, max_degree=None, weighted=True,
                           min_L=20, min_R=10, max_len=64, headline="plain_bf16", **SGNS_HP),
}
WORKLOAD = dict(BENCH["c2_youtube"])   # the reference arm's C2 configuration
# Algorithmic bytes per unit: plain SGNS pair = the context row and 1 + n output
# rows, each read and written at 4 bytes; walk draw = 16 B row bounds + 4 B
# neighbour + 4 B edge data + 4 B degree[dst], plus 4 B per footprint written.
BYTES_PER_PAIR_PLAIN = lambda d, n: 2 * (2 + n) * d * 4          # noqa: E731  context + 1+n targets, read+write
BYTES_PER_DRAW, BYTES_PER_FOOTPRINT = 28, 4
BYTES_PER_ROW_MB = lambda d: 2 * d * 2                            # noqa: E731  BF16 row, read + write
# Adjoint pass, per pair: rows read (input, positive output, negative/batch shared rows) at e bytes, the 8-byte
# fixed-point accumulators read and written by the gradient kernel, then read and cleared by the step kernel,
# which also reads and writes the row element.
BYTES_PER_PAIR_ADJOINT = lambda d, n, b, e: (2 + n / b) * d * (3 * e + 32)   # noqa: E731


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = tempfile.TemporaryFile(mode="w+")

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.seek(0)
        rows = [r for r in csv.reader(io.StringIO(self.out.read())) if len(r) >= 9]
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def reduce_max(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def make_graph_edges(workload: str = "c2_youtube"):
    from distger import graphgen
    return graphgen.chung_lu(**graphgen.CONFIGS[workload])


def ref_baseline(edges_path: str, v_num: int, rounds: int, sgns_words: int, walkers: int = 0, timeout: int = 900):
    """Runs the reference walk engine + dsgl (oracle/_ref/ref_embed) on the host cores,
    `walkers` walkers per round (0: v_num) and round 1 with the same count.
    Returns per-round walk seconds, footprints, and dsgl words / seconds."""
    import dgoracle
    exe = os.path.join(dgoracle.HERE, "_ref", "ref_embed")
    if not os.path.exists(exe):
        return None
    cores = os.cpu_count() or 1
    walk_threads = max(1, cores - 1)   # GraphEngine's worker_num = hw threads - 1 (graph.hpp:307)
    with tempfile.TemporaryDirectory() as tmp:
        cmd = [exe, "-g", edges_path, "-v", str(v_num), "-w", str(walkers or v_num), "--min_L", "20", "--min_R", "1",
               "--make-undirected", "-t", str(walk_threads), "-o", os.path.join(tmp, "w"),
               "--walk-rounds", str(rounds), "--sgns-words", str(sgns_words), "-size", "128", "-window", "10",
               "-negative", "5", "-sample", "1e-3", "-alpha", "0.01", "-iter", "1", "-min-count", "0",
               "-threads", str(cores), "-debug", "0", "-eoutput", os.path.join(tmp, "emb.txt")]
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout).stdout
    rounds_info = []
    sgns = None
    train_s = None
    for line in out.splitlines():
        if line.startswith("ref_round"):
            kv = dict(x.split("=") for x in line.split()[1:])
            rounds_info.append((float(kv["walk_s"]), int(kv["footprints"]), int(kv["walks"])))
        if "Train SGNS MPI TIME" in line:
            train_s = float(line.split(":]")[1].strip())
        if line.startswith("ref_embed"):
            kv = dict(x.split("=") for x in line.split()[1:])
            sgns = int(kv["sgns_words"])
    return {"rounds": rounds_info, "sgns_words": sgns, "sgns_train_s": train_s, "cores": cores,
            "walk_threads": walk_threads}


def pipeline_rate(walk_steps_per_s: float, words_per_s: float) -> float:
    """Footprints walked and trained per second when both stages run back to back."""
    return 1.0 / (1.0 / walk_steps_per_s + 1.0 / words_per_s)


def run_reference(args, rank, world, pg):
    """The reference's own CPU implementation of the path (walk.hpp engine + dsgl,
    oracle/_ref/ref_embed) on the host cores, on the bench workload.  It runs
    W + K walk rounds of V walkers (the engine asserts that a round visits every
    vertex, walk.hpp:723, so a round cannot be subsampled; times per round exclude
    the engine's dump and path assembly) and dsgl on the first --ref-sgns-words
    corpus tokens.  value = the pipeline rate of the two measured rates (each
    footprint walked once and trained once, as in our arm); ms_per_step = the
    measured CPU time of the K timed rounds plus the dsgl run, divided by K, so
    ms_per_step x K is time the reference actually spent."""
    if rank != 0:
        return
    wl = args.workload_bench
    w = BENCH[wl]
    form = args.mode or w["headline"]
    if wl == "c5_twitter":
        print(json.dumps({"impl": "reference", "unavailable": c5_reference_blocker(args.tmpdir)}))
        return
    from distger import graphgen
    with tempfile.TemporaryDirectory(dir=args.tmpdir) as tmp:
        path = os.path.join(tmp, "g.bin")
        graphgen.write_edges(path, make_graph_edges(wl))
        res = ref_baseline(path, w["vertices"], args.warmup + args.steps, args.ref_sgns_words,
                           timeout=args.ref_timeout)
    if res is None or len(res["rounds"]) < args.warmup + args.steps or not res["sgns_train_s"]:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_embed missing or failed "
                          "(reference walk engine + dsgl built by make -C oracle ref)"}))
        return
    timed = res["rounds"][args.warmup:]
    walk_s = sum(r[0] for r in timed)
    walk_rate = sum(r[1] - r[2] for r in timed) / walk_s
    word_rate = res["sgns_words"] / res["sgns_train_s"]
    value = pipeline_rate(walk_rate, word_rate)
    sample = (f"{len(res['rounds'])} walk rounds of {w['vertices']} walkers on the same graph "
              f"(walk.hpp internal_random_walk, {res['walk_threads']} threads; the first {args.warmup} untimed), "
              f"dsgl on the first {res['sgns_words']} corpus tokens ({res['cores']} threads)")
    cfg = {k: v for k, v in w.items() if k not in ("headline", "source")}
    cfg.update(workload=f"{wl}_{form}", sgns_form=form, walkers_per_round=w["vertices"])
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * (walk_s + res["sgns_train_s"]) / len(timed),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference", "config": cfg, "walk_steps_per_s": walk_rate, "sgns_words_per_s": word_rate,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": res["cores"], "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def host_memory_gb() -> float:
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) / 1e6
    except Exception:
        pass
    return 0.0


# Host memory the reference's engine needs for the Twitter-shaped graph: the
# records (12 B), their undirected doubling (2 x 12 B), the CSR it keeps
# (8 B per directed entry) and its co-occurrence CSR (graph.hpp:376-472, about as
# large again), plus the edge file written for it.
C5_REF_HOST_GB = 1.47e9 * (12 + 24 + 16 + 16) / 1e9 + 60


def c5_reference_blocker(tmpdir=None) -> str | None:
    """Why the reference's walk engine does not run the Twitter-shaped graph here."""
    return (f"too slow for a bench run: one walk round of the reference engine over the 41.6M walkers is "
            f"~916M footprints, at the ~3.4M steps/s it reaches on the YouTube-shaped graph on this box's cores about "
            f"4.5 minutes a round ("
            f"{3 + 5} rounds for the default warm-up and steps), after single-threaded load passes over the "
            f"1.47e9 edges and their 2.94e9 CSR entries, with about {C5_REF_HOST_GB:.0f} GB of host memory at "
            f"its peak (records, undirected doubling, CSR and co-occurrence CSR, graph.hpp:376-472, 642-824; "
            f"{host_memory_gb():.0f} GB available here)")


def cpu_baseline(args, wl, graph, host_edges):
    """The reference's own walk engine + dsgl (oracle/_ref/ref_embed) on the box's
    host cores, on a bounded sample of the same workload: one walk round of V
    walkers and dsgl on the first --ref-sgns-words corpus tokens."""
    from distger import graphgen
    w = BENCH[wl]
    with tempfile.TemporaryDirectory(dir=args.tmpdir) as tmp:
        path = os.path.join(tmp, "g.bin")
        if wl == "c5_twitter":
            return {"unavailable": c5_reference_blocker(args.tmpdir)}
        graphgen.write_edges(path, host_edges)
        walkers = w["vertices"]
        res = ref_baseline(path, w["vertices"], 1, args.ref_sgns_words, walkers=walkers, timeout=args.ref_timeout)
    if not (res and res["rounds"] and res["sgns_train_s"]):
        return {"unavailable": "oracle/_ref/ref_embed missing or failed"}
    w_s, f_, n_ = res["rounds"][0]
    cv = pipeline_rate((f_ - n_) / w_s, res["sgns_words"] / res["sgns_train_s"])
    return {"value": cv, "unit": UNIT, "cores": res["cores"], "kind": "reference",
            "sample": f"one walk round of {walkers} walkers on the same graph ({res['walk_threads']} threads) + "
                      f"dsgl on {res['sgns_words']} tokens ({res['cores']} threads)",
            "walk_steps_per_s": (f_ - n_) / w_s, "sgns_words_per_s": res["sgns_words"] / res["sgns_train_s"]}


def load_traffic():
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def build_bench_graph(workload: str, local: int):
    """The workload's graph as a device CSR.  c5_twitter: generated, deduplicated and
    built on the device (dg_edges_chung_lu, dg_graph_create_from_device_edges);
    c2_youtube, c3_livejournal: the numpy generator's records loaded through dg_graph_create_from_edges.
    Returns (graph, edge info, CSR build ms, host edges or None)."""
    import distger
    w = BENCH[workload]
    if w["source"] == "device":
        from distger.synth import EdgeList
        e = EdgeList.chung_lu(w["vertices"], w["draws"], w["exponent"], seed=0, max_degree=float(w["max_degree"]),
                              weighted=w["weighted"], device=local)
        n_edges = e.n
        torch_sync(local)
        t0 = time.perf_counter()
        graph = e.graph()
        torch_sync(local)
        build_ms = (time.perf_counter() - t0) * 1e3
        e.close()
        return graph, {"undirected_edges": n_edges}, build_ms, None
    edges = make_graph_edges(workload)
    distger.Graph(w["vertices"], edges=edges, make_undirected=True, device=local).close()   # context, module load
    t0 = time.perf_counter()
    graph = distger.Graph(w["vertices"], edges=edges, make_undirected=True, device=local)
    build_ms = (time.perf_counter() - t0) * 1e3   # host records -> device CSR with thresholds
    return graph, {"records": int(edges.size)}, build_ms, edges


def torch_sync(local: int):
    import torch
    torch.cuda.synchronize(local)


def sgns_kernel_name(form: str) -> str:
    return {"plain": "sgns_plain", "plain_bf16": "sgns_plain_bf16", "minibatch": "sgns_minibatch",
            "cbow": "sgns_cbow", "cbow_bf16": "sgns_cbow_bf16", "sg_shared": "sgns_sg_shared"}[form]


def measure_form(args, form, graph, counts, wl, rank, local, pg, with_clocks=False):
    """Warm-up and timed pipeline steps (one walk round of V walkers streamed into
    SGNS, dg_pipeline_round) of one trainer form; returns its counters, the trainer
    and the walk parameters."""
    import torch
    from distger import _lib
    from distger._lib import check, lib
    from distger.sgns import SGNS
    L = lib()
    w = BENCH[wl]
    v_num = w["vertices"]
    sgns = SGNS(v_num, counts, size=w["size"], window=w["window"], negative=w["negative"], batch_size=21,
                sample=w["sample"], alpha=w["alpha"], iter=w["iter"], min_count=w["min_count"], mode=form,
                seed=1 + rank, deterministic=2 if args.adjoint else 0, device=local,
                master_rows=args.master_rows if form in BF16_FORMS else 0)
    wp = _lib.WalkParams(min_len=w["min_L"], init_round=w["min_R"], walker_num=v_num, max_len=w["max_len"],
                         seed=2024 + rank)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")   # 256 MB > L2
    # Launch shapes timed on this workload before anything is measured (dg_walk_autotune,
    # dg_sgns_autotune), on at most 2M walkers of a round so that tuning stays short.
    tune = {}
    if not args.no_autotune:
        n_tune = min(v_num, 2_000_000)
        ti = _lib.TuneInfo()
        check(L.dg_walk_autotune(graph.handle, C.byref(wp), 2, n_tune, C.byref(ti)))
        tune["walk"] = ti.as_dict()
        ph = C.c_void_p()
        check(L.dg_walk_run_round(graph.handle, C.byref(wp), 90, n_tune, C.byref(ph)))
        ti = _lib.TuneInfo()
        check(L.dg_sgns_autotune(sgns.handle, ph, C.byref(ti)))
        tune["sgns"] = ti.as_dict()
        L.dg_paths_free(ph)

    def step(r):
        info = _lib.PipelineInfo()
        check(L.dg_pipeline_round(graph.handle, sgns.handle, C.byref(wp), r, v_num, C.c_float(0.0),
                                  C.byref(info), None))
        return info

    for i in range(args.warmup):
        step(2 + i)
    clocks = Clocks(local) if (with_clocks and rank == 0) else None
    if clocks:
        clocks.start()
    barrier(pg)
    torch.cuda.synchronize()
    l0 = L.dg_launch_count()
    acc = dict(tot_ms=0.0, walk_ms=0.0, train_ms=0.0, fp=0, steps=0, draws=0, words=0, pairs=0, rows=0)
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        info = step(2 + args.warmup + k)
        acc["tot_ms"] += info.total_ms
        acc["walk_ms"] += info.walk.walk_ms
        acc["train_ms"] += info.train.train_ms
        acc["fp"] += info.walk.footprints
        acc["steps"] += info.walk.steps
        acc["draws"] += info.walk.draws
        acc["words"] += info.train.words
        acc["pairs"] += info.train.pairs
        acc["rows"] += info.train.rows
    torch.cuda.synchronize()
    barrier(pg)
    acc["launches"] = L.dg_launch_count() - l0
    acc["clocks"] = clocks.stop() if clocks else None
    acc["tune"] = tune
    t_dev = reduce_max(pg, acc["tot_ms"] / 1e3)
    acc["t_dev"] = t_dev
    acc["value"] = reduce_sum(pg, acc["fp"]) / t_dev
    del flush
    return acc, sgns, wp


def measure_e2e(args, graph, sgns, wp, v_num, max_len, pg):
    """The same step through the reference-facing calls with host buffers: walks
    copied to pinned host memory (dg_paths_copy) and trained from there
    (dg_sgns_train_host), both copies inside the timed region."""
    import torch
    from distger import _lib
    from distger._lib import check, lib
    L = lib()
    n_walks = v_num
    h_off = torch.empty(n_walks + 1, dtype=torch.int64, pin_memory=True)
    h_verts = torch.empty(n_walks * max_len, dtype=torch.int32, pin_memory=True)
    e2e_s = 0.0
    e2e_fp = h2d = d2h = 0
    for k in range(args.steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ph = C.c_void_p()
        check(L.dg_walk_run_round(graph.handle, C.byref(wp), 100 + k, n_walks, C.byref(ph)))
        ri = _lib.RoundInfo()
        check(L.dg_paths_get_info(ph, C.byref(ri)))
        check(L.dg_paths_copy(ph, h_off.data_ptr(), h_verts.data_ptr()))
        L.dg_paths_free(ph)
        ti = _lib.TrainInfo()
        check(L.dg_sgns_train_host(sgns.handle, h_off.data_ptr(), n_walks, h_verts.data_ptr(), C.c_float(0.0),
                                   C.byref(ti)))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if k == 0:
            continue   # warm-up of the host path (allocations)
        e2e_s += dt
        e2e_fp += ri.footprints
        d2h += (n_walks + 1) * 8 + ri.footprints * 4 + 32
        h2d += (n_walks + 1) * 8 + ri.footprints * 4
    del h_off, h_verts
    return reduce_sum(pg, e2e_fp) / reduce_max(pg, e2e_s), h2d / args.steps, d2h / args.steps


def roofline(wl, form, acc, args):
    """Roofline of the dominant kernel.  achieved = the DRAM bytes the kernel moves
    per launch (ncu dram__bytes per unit measured on this workload, profiles/traffic.json,
    times the launch's units) / its CUDA-event time, so frac is the share of the
    measured copy bandwidth the kernel uses; l2_plus_dram_frac uses the access
    model's bytes instead (every row access counted, L2 hits included)."""
    hbm, peak_kind = peaks()
    traffic = load_traffic().get(wl, {})
    w = BENCH[wl]
    d, n = w["size"], w["negative"]
    if acc["train_ms"] >= acc["walk_ms"]:
        kern = sgns_kernel_name(form)
        e = 2 if form in BF16_FORMS else 4
        if form == "minibatch":
            model = acc["rows"] * 2 * d * e
        elif form in ("cbow", "cbow_bf16"):
            model = None
        elif form == "sg_shared":
            model = acc["pairs"] * 2 * d * e
        else:
            model = acc["pairs"] * 2 * (2 + n) * d * e
        if args.adjoint:
            kern = "sgns_adjoint"
            model = acc["pairs"] * BYTES_PER_PAIR_ADJOINT(d, n, 21, 4 if form == "plain" else 2)
        kms = acc["train_ms"]
        t = traffic.get(kern, {})
        measured = None
        if t.get("dram_bytes_per_pair"):
            measured = t["dram_bytes_per_pair"] * acc["pairs"]
        elif t.get("dram_bytes_per_word"):
            measured = t["dram_bytes_per_word"] * acc["words"]
    else:
        kern = "walk"
        model = acc["draws"] * BYTES_PER_DRAW + acc["fp"] * BYTES_PER_FOOTPRINT
        kms = acc["walk_ms"]
        t = traffic.get("walk", {})
        measured = t["dram_bytes_per_draw"] * acc["draws"] if t.get("dram_bytes_per_draw") else None
    sec = kms / 1e3
    per_launch = lambda x: None if x is None else x / args.steps   # noqa: E731
    roof = {"kernel": kern, "bound": "hbm", "peak": hbm, "unit": "GB/s", "peak_kind": peak_kind,
            "traffic": per_launch(measured), "traffic_source": t.get("source"),
            "model_bytes_per_launch": per_launch(model)}
    if measured is not None:
        roof["achieved"] = measured / sec / 1e9
        roof["basis"] = "measured DRAM bytes per unit (ncu) x units / kernel time"
    elif model is not None:
        roof["achieved"] = model / sec / 1e9
        roof["basis"] = "access-model bytes (L2 hits included) / kernel time"
    else:
        roof["achieved"] = None
    roof["frac"] = roof["achieved"] / hbm if roof["achieved"] else None
    if model is not None:
        roof["l2_plus_dram_frac"] = model / sec / 1e9 / hbm
    # The measured bytes of the whole step cannot outrun the copy bandwidth.
    roof["bound_check"] = "ok" if measured is None or measured / (acc["t_dev"] or 1) / 1e9 <= hbm * 1.02 \
        else "measured bytes / step time exceeds the copy bandwidth"
    return roof


def run_ours(args, rank, world, local, pg):
    import torch
    from distger import _lib

    torch.cuda.set_device(local)
    wl = args.workload_bench
    w = BENCH[wl]
    v_num = w["vertices"]
    form = args.mode or w["headline"]
    graph, einfo, graph_build_ms, host_edges = build_bench_graph(wl, local)
    out_deg, in_deg = graph.degrees()
    counts = out_deg + in_deg              # word2vec vocabulary from degrees (huge_walk.cpp:43-46)

    acc, sgns, wp = measure_form(args, form, graph, counts, wl, rank, local, pg, with_clocks=True)
    e2e_value, h2d, d2h = (None, 0, 0) if args.no_e2e else measure_e2e(args, graph, sgns, wp, v_num, w["max_len"], pg)
    sgns.close()
    roof = roofline(wl, form, acc, args)
    # FP32 plain (word2vec.cu's skip_gram_kernel rule) on the same graph, beside the headline form.
    plain = None
    if form != "plain" and not args.no_plain_leg:
        pacc, psgns, _ = measure_form(args, "plain", graph, counts, wl, rank, local, pg)
        psgns.close()
        plain = {"value": pacc["value"], "unit": UNIT, "ms_per_step": pacc["t_dev"] * 1e3 / args.steps,
                 "walk_steps_per_s": pacc["steps"] / (pacc["walk_ms"] / 1e3),
                 "sgns_words_per_s": pacc["words"] / (pacc["train_ms"] / 1e3),
                 "sgns_ms_per_step": pacc["train_ms"] / args.steps, "dtype": "f32",
                 "roofline": roofline(wl, "plain", pacc, args)}

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(args, wl, graph, host_edges)
        cfg = {k: v for k, v in w.items() if k not in ("headline", "source")}
        cfg.update(einfo)
        if form in BF16_FORMS:
            cfg["master_rows"] = args.master_rows or 65536
        cfg.update(workload=f"{wl}_{form}" + ("_adjoint" if args.adjoint else ""), sgns_form=form,
                   walkers_per_round=v_num, l2="flushed between steps (256 MB write); rows and CSR exceed L2",
                   parallelism=f"replicas x{world}")
        line = {"metric": METRIC, "value": acc["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": acc["t_dev"] * 1e3 / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "bf16" if form in BF16_FORMS else "f32",
                "data": "synthetic", "config": cfg,
                "walk_steps_per_s": acc["steps"] / (acc["walk_ms"] / 1e3),
                "sgns_words_per_s": acc["words"] / (acc["train_ms"] / 1e3),
                "walk_ms_per_step": acc["walk_ms"] / args.steps, "sgns_ms_per_step": acc["train_ms"] / args.steps,
                "footprints_per_step": acc["fp"] / args.steps, "pairs_per_step": acc["pairs"] / args.steps,
                "graph_build_ms": graph_build_ms,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": acc["launches"], "clocks": acc["clocks"], "roofline": roof, "cpu_baseline": cpu,
                "fp32_plain": plain, "autotune": acc["tune"]}
    graph.close()
    return line


AUC_HP = dict(size=128, window=10, negative=5, batch_size=21, sample=1e-3, alpha=0.01, iter=1, min_count=0)


def auc_split(workload: str):
    """The workload's graph with 10% of its edges held out (gtrain.cpp's rule) plus
    as many non-edges: (v_num, train_edges, pairs, labels)."""
    from distger import graphgen, lp
    cfg = graphgen.CONFIGS[workload]
    edges = graphgen.chung_lu(**cfg)
    train, pairs, labels = lp.split(edges, cfg["n"], frac=0.1, seed=2)
    return cfg["n"], train, pairs, labels


def run_auc_ours(args, local):
    """The whole embedding job (30 walk rounds streamed into SGNS) for each trainer
    form on the held-out split; one JSON line per form with its AUC and rates."""
    import torch
    import distger
    from distger import lp
    from distger.embed import embed
    torch.cuda.set_device(local)
    v, train, pairs, labels = auc_split(args.workload)
    runs = [(m, 0) for m in args.auc_modes.split(",")]
    if args.workers:
        runs = [(m, int(w)) for m in args.auc_modes.split(",") for w in args.workers.split(",")]
    for form, workers in runs:
        mode, _, variant = form.partition("-")          # plain, minibatch, plain-adjoint, minibatch-adjoint
        graph = distger.Graph(v, edges=train, make_undirected=True, device=local)
        clocks = Clocks(local)
        clocks.start()
        res = embed(graph, mode=mode, seed=args.seed, workers=workers, deterministic=2 if variant == "adjoint" else 0,
                    master_rows=args.master_rows, device=local, plain_shape=args.plain_shape, **AUC_HP)
        clk = clocks.stop()
        graph.close()
        m = lp.evaluate(res["embedding"], pairs, labels)
        print(json.dumps({"metric": "link-prediction AUC", "impl": "ours", "workload": args.workload,
                          "sgns_form": form, "plain_shape": args.plain_shape, "dtype": "bf16" if mode in BF16_FORMS else "f32",
                          "workers": workers or res["workers"], "master_rows": args.master_rows, "auc": m["auc"],
                          "auc_cosine": m["auc_cosine"], "test_pairs": int(labels.size), "rounds": len(res["rounds"]),
                          "embed_device_s": res["device_ms"] / 1e3, "embed_wall_s": res["rounds_wall_s"],
                          "walk_steps_per_s": res["walk_steps_per_s"], "sgns_words_per_s": res["words_per_s"],
                          "footprints": res["footprints"], "words": res["words"], "clocks": clk,
                          "config": dict(AUC_HP, split="10% edges held out + equal uniform non-edges, seed 2",
                                         walkers_per_round=v, min_L=20, min_R=5, lr="ExponentialDecayLR(alpha, 0.1)")}),
              flush=True)


def run_gcn(args, local):
    """Common-neighbour counts (the edge data the walk reads; the reference's gcn
    tool, src/tools/gcn.cpp) on the YouTube-shaped graph, undirected: the device
    kernel through the C ABI with host buffers in and out (copies timed), against
    the reference tool compiled unmodified (oracle/_ref/gcn_ref) on all host cores
    with the same edges as text.  One JSON line; `parity` compares every
    (src, dst, count) triple of the two outputs."""
    import numpy as np
    import torch
    from distger.synth import common_neighbours
    torch.cuda.set_device(local)
    edges = make_graph_edges()
    v_num = graphgen_config()["n"]
    src, dst = edges["src"], edges["dst"]
    n = int(src.size)
    common_neighbours(src, dst, v_num, device=local)   # warm-up: allocations, module load
    times = []
    for _ in range(max(args.steps, 1)):
        t0 = time.perf_counter()
        cn = common_neighbours(src, dst, v_num, device=local)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    line = {"metric": "common-neighbour counts (gcn)", "unit": "edges/s", "impl": "ours", "value": n / t,
            "ms_per_call": t * 1e3, "calls": len(times), "higher_is_better": True,
            "config": {"graph": "youtube-shaped chung-lu", "vertices": v_num, "undirected_edges": n,
                       "make_undirected": True, "buffers": "host in, host out (copies inside the timed call)"}}
    import dgoracle
    tool = os.path.join(dgoracle.HERE, "_ref", "gcn_ref")
    if not os.path.exists(tool):
        line["reference"] = {"unavailable": "oracle/_ref/gcn_ref not built (make -C oracle ref)"}
    else:
        import pandas as pd
        cores = os.cpu_count() or 1
        with tempfile.TemporaryDirectory(dir=args.tmpdir) as tmp:
            inp, outp = os.path.join(tmp, "e.txt"), os.path.join(tmp, "o.txt")
            pd.DataFrame({"s": src, "d": dst}).to_csv(inp, sep=" ", header=False, index=False)
            t0 = time.perf_counter()
            r = subprocess.run([tool, "-i", inp, "-o", outp, "-v", str(v_num), "-t", str(cores), "-s", "unweighted",
                                "--make-undirected"], capture_output=True, text=True, timeout=args.ref_timeout)
            tr = time.perf_counter() - t0
            if r.returncode != 0:
                line["reference"] = {"unavailable": f"gcn_ref exited {r.returncode}"}
            else:
                ref = pd.read_csv(outp, sep=" ", header=None).to_numpy(np.int64)
                ours = np.stack([src.astype(np.int64), dst.astype(np.int64), cn.astype(np.int64)], axis=1)
                same = ref.shape == ours.shape and np.array_equal(ref[np.lexsort(ref.T[::-1])],
                                                                    ours[np.lexsort(ours.T[::-1])])
                line["reference"] = {"value": n / tr, "unit": "edges/s", "cores": cores, "kind": "reference",
                                     "seconds": tr, "note": "wall time of the tool: text read, counts, text write"}
                line["parity"] = "identical (src, dst, count) triples on all edges" if same else "DIFFERS"
    print(json.dumps(line))


def graphgen_config():
    from distger import graphgen
    return graphgen.CONFIGS["c2_youtube"]


def run_auc_reference(args):
    """The reference walk engine + dsgl (oracle/_ref/ref_embed) on the same split,
    all 30 rounds and the whole corpus, embedding scored by the same AUC code."""
    import dgoracle
    from distger import graphgen, lp
    exe = os.path.join(dgoracle.HERE, "_ref", "ref_embed")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_embed not built"}))
        return
    v, train, pairs, labels = auc_split(args.workload)
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory(dir=args.tmpdir) as tmp:
        path = os.path.join(tmp, "g.bin")
        graphgen.write_edges(path, train)
        emb_path = os.path.join(tmp, "emb.txt")
        cmd = [exe, "-g", path, "-v", str(v), "-w", str(v), "--min_L", "20", "--min_R", "5", "--make-undirected",
               "-t", str(max(1, cores - 1)), "-o", os.path.join(tmp, "w"), "-size", "128", "-window", "10",
               "-negative", "5", "-sample", "1e-3", "-alpha", "0.01", "-iter", "1", "-min-count", "0",
               "-threads", str(cores), "-debug", "0", "-eoutput", emb_path]
        t0 = time.perf_counter()
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=args.ref_timeout).stdout
        wall = time.perf_counter() - t0
        kv = {}
        for line in out.splitlines():
            if line.startswith("ref_embed"):
                kv = dict(x.split("=") for x in line.split()[1:])
        emb = lp.read_embedding_text(emb_path, v)
    m = lp.evaluate(emb, pairs, labels)
    walk_s, sgns_s = float(kv.get("walk_s", "nan")), float(kv.get("sgns_s", "nan"))
    fp, walks, words = int(kv.get("footprints", 0)), int(kv.get("walks", 0)), int(kv.get("sgns_words", 0))
    print(json.dumps({"metric": "link-prediction AUC", "impl": "reference", "workload": args.workload,
                      "sgns_form": "dsgl", "dtype": "f32", "auc": m["auc"], "auc_cosine": m["auc_cosine"],
                      "test_pairs": int(labels.size), "rounds": int(kv.get("rounds", 0)), "walk_s": walk_s,
                      "sgns_s": sgns_s, "embed_wall_s": wall, "walk_steps_per_s": (fp - walks) / walk_s,
                      "sgns_words_per_s": words / sgns_s, "footprints": fp, "words": words, "cores": cores,
                      "config": dict(AUC_HP, split="10% edges held out + equal uniform non-edges, seed 2",
                                     walkers_per_round=v, min_L=20, min_R=5)}), flush=True)


# Graphs generated, split and built on the device (dg_edges_chung_lu, dg_edges_split,
# dg_graph_create_from_device_edges); scored by dg_lp_auc.
# C5: 2.417e9 draws leave ~1.47e9 unique undirected pairs (hub pairs repeat; measured
# 2.3e9 -> 1.395e9, 2.7e9 -> 1.652e9 unique).
SYNTH = {
    "c5_twitter": dict(n=41_652_230, m=2_417_000_000, beta=1.9, max_degree=3_000_000.0, weighted=False,
                       holdout=0.01, min_r=5),
    "c2_youtube_device": dict(n=1_138_499, m=2_990_443, beta=2.1, max_degree=28_000.0, weighted=True,
                              holdout=0.1, min_r=5),
}


def run_auc_synth(args, local):
    """The whole job on a device-generated graph: generate, hold out, build the CSR,
    walk + train --rounds rounds per form, score on the device.  One JSON line per form."""
    import torch
    from distger.embed import embed
    from distger.synth import EdgeList
    torch.cuda.set_device(local)
    cfg = SYNTH[args.workload]
    runs = [(f, 0) for f in args.auc_modes.split(",")]
    if args.workers:
        runs = [(f, int(w)) for f in args.auc_modes.split(",") for w in args.workers.split(",")]
    for form, workers in runs:
        mode, _, variant = form.partition("-")
        t0 = time.perf_counter()
        e = EdgeList.chung_lu(cfg["n"], cfg["m"], cfg["beta"], seed=0, max_degree=cfg["max_degree"],
                              weighted=cfg["weighted"], device=local)
        t1 = time.perf_counter()
        n_edges = e.n
        pairs = e.split(cfg["holdout"], seed=2)
        t2 = time.perf_counter()
        graph = e.graph()
        t3 = time.perf_counter()
        e.close()
        clocks = Clocks(local)
        clocks.start()
        res = embed(graph, mode=mode, seed=args.seed, rounds=args.rounds, init_round=cfg["min_r"], max_len=32,
                    deterministic=2 if variant == "adjoint" else 0, workers=workers, master_rows=args.master_rows,
                    keep_trainer=True, device=local, plain_shape=args.plain_shape, **AUC_HP)
        clk = clocks.stop()
        t4 = time.perf_counter()
        sgns = res.pop("trainer")
        m = pairs.auc(sgns)
        t5 = time.perf_counter()
        print(json.dumps({"metric": "link-prediction AUC", "impl": "ours", "workload": args.workload,
                          "sgns_form": form, "plain_shape": args.plain_shape, "dtype": "bf16" if mode in BF16_FORMS else "f32", "workers": res["workers"],
                          "master_rows": args.master_rows,
                          "auc": m["auc"], "auc_cosine": m["auc_cosine"], "test_pairs": pairs.n_pos + pairs.n_neg,
                          "vertices": cfg["n"], "undirected_edges": n_edges, "rounds": len(res["rounds"]),
                          "generate_s": t1 - t0, "split_s": t2 - t1, "csr_build_s": t3 - t2,
                          "embed_device_s": res["device_ms"] / 1e3, "embed_wall_s": res["wall_s"],
                          "score_s": t5 - t4, "end_to_end_s": t5 - t0,
                          "walk_steps_per_s": res["walk_steps_per_s"], "sgns_words_per_s": res["words_per_s"],
                          "footprints": res["footprints"], "words": res["words"], "clocks": clk,
                          "config": dict(AUC_HP, graph=dict(cfg), split_seed=2, walkers_per_round=cfg["n"],
                                         min_L=20, lr="ExponentialDecayLR(alpha, 0.1)",
                                         note="rounds 1..%d of 30" % args.rounds)}), flush=True)
        sgns.close()
        pairs.close()
        graph.close()


def run_profile_case(args, local):
    """A short case of one kernel for ncu: the --profile-workload graph and trainer,
    one walk round of --profile-walks walkers (0: all V), then one SGNS launch over
    those walks.  Prints a one-line summary.  On the YouTube-shaped graph the rows
    exceed L2 already at 50,000 walks; the Twitter-shaped graph is for one-pass
    metrics only (it holds tens of GB on the device)."""
    from distger import _lib
    from distger._lib import check, lib
    from distger.sgns import SGNS
    L = lib()
    wl = args.profile_workload
    w = BENCH[wl]
    v_num = w["vertices"]
    graph, _, _, _ = build_bench_graph(wl, local)
    od, idg = graph.degrees()
    counts = od + idg
    walkers = args.profile_walks or v_num
    wp = _lib.WalkParams(min_len=w["min_L"], init_round=w["min_R"], walker_num=v_num, max_len=w["max_len"], seed=7)
    p1 = C.c_void_p()
    check(L.dg_walk_run_round(graph.handle, C.byref(wp), 2, walkers, C.byref(p1)))
    ri = _lib.RoundInfo()
    check(L.dg_paths_get_info(p1, C.byref(ri)))
    out = {"case": args.profile, "workload": wl, "walks": walkers, "walk_ms": ri.walk_ms, "draws": ri.draws,
           "footprints": ri.footprints}
    if args.profile in ("sgns", "sgns_bf16", "minibatch", "adjoint", "cbow", "cbow_bf16", "sg_shared"):
        pmode = {"minibatch": "minibatch", "sgns_bf16": "plain_bf16", "cbow": "cbow", "cbow_bf16": "cbow_bf16",
                 "sg_shared": "sg_shared"}.get(args.profile, "plain")
        s = SGNS(v_num, counts, size=w["size"], window=w["window"], negative=w["negative"], batch_size=21,
                 sample=w["sample"], alpha=w["alpha"], iter=1, min_count=0, mode=pmode, seed=1,
                 deterministic=2 if args.profile == "adjoint" else 0, device=local)
        ti = _lib.TrainInfo()
        check(L.dg_sgns_train_paths(s.handle, p1, C.c_float(0.0), C.byref(ti)))
        out.update({"train_ms": ti.train_ms, "pairs": ti.pairs, "words": ti.words})
        s.close()
    L.dg_paths_free(p1)
    graph.close()
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile", choices=["walk", "sgns", "sgns_bf16", "minibatch", "adjoint", "cbow", "cbow_bf16",
                                          "sg_shared"],
                    default=None, help="run one launch of a kernel for ncu and exit")
    ap.add_argument("--profile-walks", type=int, default=50_000, help="--profile: walkers of the round (0: all)")
    ap.add_argument("--profile-workload", choices=sorted(BENCH), default="c2_youtube")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["plain", "plain_bf16", "minibatch", "cbow", "cbow_bf16", "sg_shared"], default=None,
                    help="trainer form of the bench line (default: the workload's headline form)")
    ap.add_argument("--bench-workload", dest="workload_bench", choices=sorted(BENCH), default="c5_twitter")
    ap.add_argument("--no-plain-leg", action="store_true", help="skip the FP32 plain measurement beside the headline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer (e2e) measurement (experiments only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--adjoint", action="store_true", help="train by adjoint gradient steps (deterministic mode 2)")
    ap.add_argument("--ref-sgns-words", type=int, default=1_000_000)
    ap.add_argument("--auc", action="store_true",
                    help="run the whole embedding job on a 10%%-held-out split and print link-prediction AUC lines")
    ap.add_argument("--workload", choices=["c1_small", "c2_youtube", "c3_livejournal", "c5_twitter",
                                           "c2_youtube_device"], default="c1_small",
                    help="graph of the --auc run (c5_twitter and *_device: generated and split on the device)")
    ap.add_argument("--rounds", type=int, default=30, help="--auc on device-generated graphs: walk rounds")
    ap.add_argument("--auc-modes", default="plain,minibatch")
    ap.add_argument("--gcn", action="store_true",
                    help="time the common-neighbour precompute against the reference gcn tool and exit")
    ap.add_argument("--plain-shape", type=int, default=None,
                    help="AUC runs: launch shape of the plain kernel (an index of the autotuner's list)")
    ap.add_argument("--workers", default="", help="--auc: comma-separated trainer worker counts to sweep (0 = auto)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--master-rows", type=int, default=0,
                    help="FP32 master rows (hottest words) of the BF16 forms; 0 = 65,536")
    ap.add_argument("--tmpdir", default=None)
    ap.add_argument("--ref-timeout", type=int, default=7200)
    args = ap.parse_args()
    if args.profile:
        run_profile_case(args, int(os.environ.get("LOCAL_RANK", "0")))
        return
    if args.gcn:
        run_gcn(args, int(os.environ.get("LOCAL_RANK", "0")))
        return
    if args.auc:
        if args.impl == "reference":
            run_auc_reference(args)
        elif args.workload in SYNTH:
            run_auc_synth(args, int(os.environ.get("LOCAL_RANK", "0")))
        else:
            run_auc_ours(args, int(os.environ.get("LOCAL_RANK", "0")))
        return
    rank, world, local, pg = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, rank, world, pg)
        else:
            line = run_ours(args, rank, world, local, pg)
            if rank == 0 and line is not None:
                print(json.dumps(line))
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
