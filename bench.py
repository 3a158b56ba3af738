#!/usr/bin/env python
"""Benchmark of the block-Wiedemann Krylov step on B200.

Workload (the large single-matrix configuration): a 2,000,000 x 1,500,000 CSR
matrix over p = 2013265921 with 12 distinct Zipf(1.1) columns per row, values
uniform in [1, p-1] and 10,000 duplicated rows, seeded synthetic data; block
width b = 16.  One step = one application of B = D_c A^T D_r A D_c (two SpMMs)
together with the two fused sequence terms S_{2k+1}, S_{2k+2}.

Metric: Krylov SpMM HBM GB/s on the algorithmic byte count per application
    sum over {A, A^T} of (8 nnz + 4 (rows + 1)) + 4 b 2 (m + n)
(CSR read once, dense blocks read and written once).  The working set
(~0.7 GB) is far larger than the 126 MB L2, so no explicit flush is needed.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N > 1 runs independent replicas (one matrix per GPU, no collective on the
data path); value is the total over all ranks, time the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

P = 2013265921
METRIC = "Krylov SpMM HBM GB/s"
WORKLOAD = "zipf_2000000x1500000_nnz12_b16"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--b", type=int, default=16)
    ap.add_argument("--small", action="store_true", help="scaled-down workload for quick checks")
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the full matrix size (profiling runs)")
    ap.add_argument("--no-rank", action="store_true", help="skip the rank-pipeline measurement")
    ap.add_argument("--cpu-samples", type=int, default=6)
    return ap.parse_args()


def workload(small: bool, scale: float = 1.0):
    from rust_rank_b200 import synth

    if small:
        scale = 0.1
    if scale != 1.0:
        return synth.zipf_large(m=int(2_000_000 * scale), n=int(1_500_000 * scale), k=12,
                                dup_rows=int(10_000 * scale), p=P, seed=44)
    return synth.zipf_large(p=P, seed=44)


def dist_init(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """Max of x over the ranks (device tensor under NCCL, host tensor under gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, bytes_per_app: float, apps: int, ms_max: float) -> float:
    """Whole-job GB/s of `world` replicas that each ran `apps` applications;
    the slowest rank's time (ms_max) is the job's time."""
    return world * bytes_per_app * apps / (ms_max / 1e3) / 1e9


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def bench_config(args, m, n, nnz, world):
    """The `config` dict of the JSON line; both arms print the same one."""
    full = args.scale == 1.0 and not args.small
    return {"workload": WORKLOAD if full else f"{WORKLOAD}_scaled", "m": m, "n": n, "nnz": int(nnz), "b": args.b,
            "p": P, "parallelism": f"replicas x{world}", "l2_policy": "inputs larger than L2 (working set ~0.7 GB)"}


def cpu_baseline(rowptr, col, val, m, n, b, samples):
    """The oracle (CPU restatement of the reference's Krylov worker + consumer) on the same matrix."""
    import oracle
    from rust_rank_b200 import synth

    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    dr, dc = synth.preconditioners(m, n, P, 1)
    V = synth.random_vectors(b, n, P, 2)
    op = oracle.KrylovOp(rowptr, col, val, m, n, P, dr, dc, V)
    op.step()  # warm-up
    t0 = time.perf_counter()
    for _ in range(samples):
        op.step()
    dt = (time.perf_counter() - t0) / samples
    op.close()
    bytes_app = 2 * (8.0 * rowptr[-1]) + 4.0 * (m + 1) + 4.0 * (n + 1) + 4.0 * b * 2 * (m + n)
    return bytes_app / dt / 1e9, dt, threads


def run_reference(args):
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    rowptr, col, val, m, n = workload(args.small, args.scale)
    import oracle
    from rust_rank_b200 import synth

    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    dr, dc = synth.preconditioners(m, n, P, 1)
    V = synth.random_vectors(args.b, n, P, 2)
    op = oracle.KrylovOp(rowptr, col, val, m, n, P, dr, dc, V)
    for _ in range(args.warmup):
        op.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        op.step()
    dt = time.perf_counter() - t0
    bytes_app = 2 * (8.0 * rowptr[-1]) + 4.0 * (m + 1) + 4.0 * (n + 1) + 4.0 * args.b * 2 * (m + n)
    v = bytes_app * args.steps / dt / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 mod p (u64/u128 accum)",
        "data": "synthetic (seeded)",
        "config": bench_config(args, m, n, rowptr[-1], int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} applications of B on the full matrix"},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "CPU restatement of the reference Rust path (the reference cannot be built here: no Rust toolchain)",
    }
    print(json.dumps(line), flush=True)


def rank_pipeline(ctx, reps=3):
    """Whole rank computation (Krylov + PM-basis + readout) on the plain single-matrix config."""
    import rust_rank_b200 as rr
    from rust_rank_b200 import synth

    rowptr, col, val, m, n = synth.plain_single(n=20000, k=6, dep_rows=500, p=P, seed=43)
    a = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n)
    dm = a.to_device(P, ctx)
    b = 8
    rp, cp = synth.preconditioners(m, n, P, 5)
    V = synth.random_vectors(b, n, P, 6)
    rank = rr.block_wiedemann_rank(dm, b, P, row_precond=rp, col_precond=cp, v=V, ctx=ctx)  # warm-up
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        r = rr.block_wiedemann_rank(dm, b, P, row_precond=rp, col_precond=cp, v=V, ctx=ctx)
        times.append(time.perf_counter() - t0)
        assert r == rank
    med = statistics.median(times)
    return {"workload": "plain_20000x20000_nnz6_b8 (500 dependent rows)", "rank": rank,
            "upper_bound_by_construction": m - 500, "ms_per_rank": 1e3 * med, "ranks_per_sec": 1.0 / med,
            "timing": "wall clock of rr_rank on a resident matrix, median of %d" % reps}


def batched_vs_plain(ctx, nmat=256, rmin=1000, rmax=200_000, b=16, workers=4, runs=1):
    """Graph-complex-like batch (rows log-uniform, cols = rows * U(0.6, 1), 3..10
    entries +-1 per row, planted deficits): the batched engine (rr_batch_*)
    against the plain one-matrix-at-a-time GPU loop (rr_rank) on the same set."""
    import rust_rank_b200 as rr
    from rust_rank_b200 import synth

    mats = synth.graph_complex_batch(nmat=nmat, rmin=rmin, rmax=rmax)
    drs, dcs, vs = [], [], []
    for i, (_, _, _, m, n) in enumerate(mats):
        dr, dc = synth.preconditioners(m, n, P, 100 + 10 * i)
        drs.append(dr)
        dcs.append(dc)
        vs.append(synth.random_vectors(b, n, P, 101 + 10 * i))
    # untimed warm-up of both modes (module loading, memory-pool growth)
    w = list(range(0, nmat, 6))
    wb = rr.Batch([mats[i] for i in w], b, P, [drs[i] for i in w], [dcs[i] for i in w], [vs[i] for i in w], ctx)
    wb.ranks(workers)
    wb.close()
    for i in w[:2]:
        rr.block_wiedemann_rank(rr.CsrMatrix.from_arrays(*mats[i]).to_device(P, ctx), b, P, row_precond=drs[i],
                                col_precond=dcs[i], v=vs[i], ctx=ctx)
    # the batched time varies from run to run (host threads, generator
    # scheduling): the median of `runs` runs is reported, with all of them
    t_runs = []
    for _ in range(runs):
        t0 = time.perf_counter()
        bt = rr.Batch(mats, b, P, drs, dcs, vs, ctx)
        ranks = bt.ranks(workers)
        t_runs.append(time.perf_counter() - t0)
        bt.close()
    t_batch = statistics.median(t_runs)
    t0 = time.perf_counter()
    plain = []
    for i, (rowptr, col, val, m, n) in enumerate(mats):
        dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(P, ctx)
        plain.append(rr.block_wiedemann_rank(dm, b, P, row_precond=drs[i], col_precond=dcs[i], v=vs[i], ctx=ctx))
        dm.close()
    t_plain = time.perf_counter() - t0
    assert list(ranks) == plain, "batched ranks differ from the plain loop"
    shapes = []
    bt = rr.Batch(mats[: min(nmat, 8)], b, P, drs[:8], dcs[:8], vs[:8], ctx)
    shapes = [{"apps_from": a, "ctas": c, "lanes_per_thread": l, "rows_per_warp": r}
              for (a, c), (l, r) in zip(bt.tuning(), bt.tuning_shape())]
    bt.close()
    return {"workload": f"graph_complex_batch_{nmat}_rows_{rmin}-{rmax}_b{b}",
            "matrices": nmat, "batched_ranks_per_sec": nmat / t_batch, "plain_ranks_per_sec": nmat / t_plain,
            "tuned_shapes_first8": shapes,
            "batched_over_plain": t_plain / t_batch, "batched_s": t_batch, "batched_runs_s": t_runs,
            "plain_s": t_plain,
            "timing": "wall clock, host matrices in, ranks out (upload, Krylov, generator, readout), after one "
                  "untimed warm-up of both modes on a subset; batched: median of %d run(s)" % runs}


def served_stream(nreq=12, rmin=10_000, rmax=2_000_000, rate=50.0, b=16, seed=48):
    """Poisson arrivals (mean `rate` req/s) of rank requests (rows log-uniform,
    4..12 entries +-1 per row) through the rank service (rr_server_*), against
    the plain sequential GPU loop on the same requests."""
    import threading

    import rust_rank_b200 as rr
    from rust_rank_b200 import synth

    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(nreq):
        m = int(np.exp(rng.uniform(np.log(rmin), np.log(rmax))))
        n = max(3, int(m * rng.uniform(0.6, 1.0)))
        rowptr, col, val, m, n = synth.incidence_fast(m, n, 4, 12, n // 100 if i % 5 == 0 else 0, P, seed * 1000 + i)
        dr, dc = synth.preconditioners(m, n, P, seed + 3 * i)
        reqs.append((rowptr, col, val, m, n, dr, dc, synth.random_vectors(b, n, P, seed + 3 * i + 1)))
    gaps = rng.exponential(1.0 / rate, size=nreq)
    # untimed warm-up (contexts, module loading, memory-pool growth)
    srv = rr.Server(b, P, lanes=4, workers=8, max_active=32, chunk_apps=64)
    for r in reqs[:3]:
        srv.result(srv.submit(*r[:3], r[3], r[4], *r[5:]), timeout=600.0)
    srv.close()
    srv = rr.Server(b, P, lanes=4, workers=8, max_active=32, chunk_apps=64)
    ids = [None] * nreq

    def submitter():
        t_next = time.perf_counter()
        for i, r in enumerate(reqs):
            t_next += gaps[i]
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            ids[i] = srv.submit(*r[:3], r[3], r[4], *r[5:])

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    served = [srv.result(i, timeout=600.0)[0] for i in ids]
    st = srv.stats()
    srv.close()
    ctx = rr.Context(0)
    t0 = time.perf_counter()
    plain = []
    for r in reqs:
        dm = rr.CsrMatrix.from_arrays(*r[:3], r[3], r[4]).to_device(P, ctx)
        plain.append(rr.block_wiedemann_rank(dm, b, P, row_precond=r[5], col_precond=r[6], v=r[7], ctx=ctx))
        dm.close()
    t_plain = time.perf_counter() - t0
    ctx.close()
    assert served == plain, "served ranks differ from the plain loop"
    return {"workload": f"served_poisson_{rate:g}rps_{nreq}req_rows_{rmin}-{rmax}_nnz4-12_b{b}",
            "requests": nreq, "served_ranks_per_sec": st["ranks_per_s"], "p50_ms": st["p50_ms"],
            "p99_ms": st["p99_ms"], "plain_ranks_per_sec": nreq / t_plain,
            "served_over_plain": st["ranks_per_s"] / (nreq / t_plain),
            "timing": "latency = submit to rank (queueing included); throughput = completions / (last completion - "
                      "first submit); plain = sequential upload + rr_rank per request; one untimed warm-up service run"}


def full_rank_zipf(ctx, rowptr, col, val, m, n, b=16):
    """Host CSR in, rank out on the large Zipf matrix: rr_matrix_create (device
    build), the Krylov sequence of the stated length N/b + N/b + 32 (N = the
    smaller dimension) -- which the rank path, like src/main.rs:500-503, rounds
    up to the next power of two for b > 1 -- the PM-basis of order d = largest
    power of two <= length, and the rank readout, all through the public API,
    timed by wall clock."""
    import rust_rank_b200 as rr
    from rust_rank_b200 import synth

    dr, dc = synth.preconditioners(m, n, P, 61)
    V = synth.random_vectors(b, n, P, 62)
    L = 2 * (min(m, n) // b) + 32
    t0 = time.perf_counter()
    dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(P, ctx)
    t1 = time.perf_counter()
    rank = rr.block_wiedemann_rank(dm, b, P, row_precond=dr, col_precond=dc, v=V, max_nlen=L, ctx=ctx)
    t2 = time.perf_counter()
    dm.close()
    nonempty = int(np.count_nonzero(np.bincount(col, minlength=n)))
    L2 = 1 << (L - 1).bit_length() if b > 1 else L  # src/main.rs:500-503
    return {"workload": f"zipf_{m}x{n}_nnz{int(rowptr[-1])}_b{b}", "stated_length": L, "sequence_terms": L2 + 1,
            "applications_of_B": L2 // 2, "generator_order": L2, "rank": rank,
            "upper_bound_nonempty_columns": nonempty, "s_total": t2 - t0, "s_matrix_build": t1 - t0,
            "ranks_per_sec": 1.0 / (t2 - t0),
            "timing": "wall clock, host CSR in (pageable numpy arrays), rank out"}


def pm_basis_stage(ctx, b=16, ds=(1 << 14, 1 << 16)):
    """PM-basis alone on 2b x 2b generators of uniform random sequences."""
    import rust_rank_b200 as rr

    out = {}
    rng = np.random.default_rng(4)
    for d in ds:
        seq = rng.integers(0, P, size=(b * (b + 1) // 2, d + 1), dtype=np.int64).astype(np.uint32)
        for tc in (True, False):
            ctx.set_pm_tensor_cores(tc)
            best, ref = None, None
            for _ in range(2):  # the first call also grows the memory pool to this size's workspace
                t0 = time.perf_counter()
                M, delta = rr.PM_Basis(seq, d, P, ctx)
                dt = time.perf_counter() - t0
                best = dt if best is None else min(best, dt)
            out[f"d{d}_ms" if tc else f"d{d}_cuda_core_ms"] = 1e3 * best
        ctx.set_pm_tensor_cores(True)
    for p_small in (3323,):  # a prime without a suitable NTT: products by CRT over NTT primes
        d = ds[0]
        seq = rng.integers(0, p_small, size=(b * (b + 1) // 2, d + 1), dtype=np.int64).astype(np.uint32)
        best = None
        for _ in range(2):
            t0 = time.perf_counter()
            rr.PM_Basis(seq, d, p_small, ctx)
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        out[f"d{d}_p{p_small}_ms"] = 1e3 * best
    out["workload"] = f"pm_basis_b{b}_2b{2 * b}_uniform_random_seq"
    out["contractions"] = ("dN_ms: leaf residual updates and block-basis products on the int8 tensor cores "
                           "(byte limbs, exact); dN_cuda_core_ms: the same on the CUDA cores (64-bit sums)")
    out["timing"] = "wall clock of rr_pm_basis (host sequence in, generator out), best of 2"
    return out


def run_engine(args):
    import torch

    import rust_rank_b200 as rr
    from rust_rank_b200 import synth

    world, rank, local = dist_init(args.gpus)
    ctx = rr.Context(local)
    rowptr, col, val, m, n = workload(args.small, args.scale)
    b = args.b
    dr, dc = synth.preconditioners(m, n, P, 1)
    V = synth.random_vectors(b, n, P, 2)
    t0 = time.perf_counter()
    dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(P, ctx)
    setup_s = time.perf_counter() - t0
    ks = rr.KrylovStream(dm, V, dr, dc, 0)
    bytes_app = ks.bytes_per_application()
    ks.step_device(args.warmup)
    ctx.synchronize()

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = ks.launch_count()
    with ClockSampler(local) as clk:
        barrier(world)
        ctx.synchronize()
        e0.record(stream)
        ks.step_device(args.steps)
        e1.record(stream)
        ctx.synchronize()
        barrier(world)
    launches = ks.launch_count() - launches0
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world)
    clocks = clk.summary()
    value = replica_throughput(world, bytes_app, args.steps, ms_max)

    # per-phase device times (CUDA events on the context stream, inside the library)
    ph = ks.profile(max(4, min(args.steps, 10)))
    pb = ks.phase_bytes()
    traffic = ncu_traffic()
    peak, peak_kind = measured_peak()
    # dominant kernel: the pass over A^T when chunked rows exist is two launches; report each phase
    phases = {
        "pass_A": {"ms": ph[0], "alg_bytes": pb[0], "gbs": pb[0] / (ph[0] / 1e3) / 1e9},
        "pass_At_chunks+rows": {"ms": ph[1] + ph[2], "alg_bytes": pb[1], "gbs": pb[1] / ((ph[1] + ph[2]) / 1e3) / 1e9,
                                "chunk_ms": ph[1], "rows_ms": ph[2]},
    }
    dom = max(phases, key=lambda k: phases[k]["ms"])
    ach = phases[dom]["gbs"]
    roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_kind": peak_kind, "traffic": traffic.get(dom), "phases": phases}

    # e2e: the public API with host buffers (pinned V / preconditioners in, terms + final block out)
    def pinned(a):
        return torch.from_numpy(a.view(np.int32)).pin_memory().numpy().view(np.uint32)

    Vp, drp, dcp = pinned(V), pinned(dr), pinned(dc)
    np_ = b * (b + 1) // 2
    seq = torch.zeros((np_, 2 * args.steps + 2), dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    curv_out = torch.zeros((b, n), dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    host_csr = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n)
    csr_bytes = rowptr.nbytes + col.nbytes + val.nbytes
    # whole job through the public API: host CSR in (device build of the
    # degree-ordered CSR and its transpose), sequence and final block out
    barrier(world)
    t0 = time.perf_counter()
    dm2 = host_csr.to_device(P, ctx)
    t_build = time.perf_counter() - t0
    ks2 = rr.KrylovStream(dm2, Vp, drp, dcp, 0)
    L = ks2.advance(2 * args.steps, seq)
    ks2.get_curv(out=curv_out)
    ks2.close()
    dm2.close()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, world)
    assert L == 2 * args.steps + 1
    # the same on the resident matrix (the part after the build)
    barrier(world)
    t0 = time.perf_counter()
    ks3 = rr.KrylovStream(dm, Vp, drp, dcp, 0)
    L3 = ks3.advance(2 * args.steps, seq)
    ks3.get_curv(out=curv_out)
    res_s = max_over_ranks(time.perf_counter() - t0, world)
    assert L3 == L
    ks3.close()
    e2e = {"value": replica_throughput(world, bytes_app, args.steps, 1e3 * e2e_s), "unit": "GB/s",
           "h2d_bytes_per_step": (csr_bytes + V.nbytes + dr.nbytes + dc.nbytes) / args.steps,
           "d2h_bytes_per_step": (4.0 * np_ * L + curv_out.nbytes) / args.steps,
           "matrix_build_s": t_build,
           "resident_matrix_value": replica_throughput(world, bytes_app, args.steps, 1e3 * res_s),
           "timing": "wall clock over rr_matrix_create (host CSR in, device build) + rr_krylov_create + "
                     "rr_krylov_advance + rr_krylov_get_curv + destroy; resident_matrix_value: the same "
                     "without rr_matrix_create"}

    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 mod p (u64 lazy accum)", "data": "synthetic (seeded)",
        "config": bench_config(args, m, n, rowptr[-1], world),
        "roofline": roof, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
        "matrix_setup_s": setup_s,
    }
    ks.close()
    dm.close()
    # the GPU pipelines first, the CPU baseline last: its thread pool would
    # otherwise share the host cores with the engine's host threads
    if rank == 0 and world == 1 and not args.no_rank:
        line["rank_pipeline"] = rank_pipeline(ctx)
        line["pm_basis"] = pm_basis_stage(ctx)
        line["full_rank"] = full_rank_zipf(ctx, rowptr, col, val, m, n, b)
        line["batched"] = batched_vs_plain(ctx)
        line["served"] = served_stream()
    if rank == 0 and world == 1 and args.cpu_samples > 0:
        v, dt, threads = cpu_baseline(rowptr, col, val, m, n, b, args.cpu_samples)
        line["cpu_baseline"] = {"value": v, "unit": "GB/s", "cores": threads, "kind": "port",
                                "sample": f"{args.cpu_samples} applications of B (with both sequence terms) on the "
                                          "full matrix, oracle restatement of the reference CPU path"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
