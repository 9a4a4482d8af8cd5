"""Benchmark of the B200 BorderedCR solver on the headline BABD workload.

Workload (one "step" = factorize + solve of one system):
  trapezoid-collocation BABD, n=16, nblock=100000, qr=qx=2, nr=nx=4, one
  right-hand side, FP64, internal LU, last block LU (seeded synthetic data).
  unknowns = ncols = 16*100001 + 2 + 4 = 1,600,022.

  value : ncols / (device time of factorize + solve), matrix resident in HBM
  e2e   : the same metric through the C ABI with host buffers
          (bcr_factorize uploads the matrix from pinned host memory,
           bcr_solve copies the right-hand side in and the solution out)

  variants: every other workload of the benchmark plan, each through its own
          CUDA graph, device-timed: n=8 nblock=1000 (the CPU-sized case); this
          workload with the QR panel, with 8 right-hand sides and on the mixed
          path (FP32 factors + FP64 refinement to rel. residual <= 1e-12); FP64
          and mixed on n=32, nblock=65536, nr=nx=8 at kappa = 1, 10, 100 and on
          n=128, nblock=8192, qr=qx=4, nr=nx=16 (the mixed pair kernel there
          runs its products on the tcgen05 tensor cores); a batch of 4096
          uneven systems (systems/s, p50/p99 of the batch latency; one launch
          per level, and for comparison one persistent launch per class with a
          per-system level schedule); and the reference's own
          BorderedCR<float> (unrefined FP32) on this workload.

  accuracy: every entry carries its relative residual
          ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf), with A x taken by
          the reference's own Mv on the host, and its forward error
          ||x - x_ref||_inf / ||x_ref||_inf against the reference BorderedCR's
          solution of the same seeded system (oracle/_ref, the unmodified
          reference sources), whose host-core time is reported beside it.

The matrix (0.65 GB) is larger than L2 (126 MB), so no L2 flush is needed
between steps.  Multi-GPU: one process per GPU, each solving its own system
(independent replicas, weak scaling, no collective on the data path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
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

METRIC = "BABD factor+solve unknowns/s at rel. residual ≤1e-12: mixed vs plain FP64 GPU"
# DRAM bytes per block moved by the factorization kernels of this workload,
# from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of the
# same workload at nblock=40000 (the traffic grows with the blocks)
FACT_DRAM_BYTES_PER_BLOCK = 21542
CFG = dict(nblock=100000, n=16, qr=2, qx=2, nr=4, nx=4)


def workload_config(extra=None):
    c = {"workload": "trapezoid-collocation BABD n=16 nblock=100000 qr=qx=2 nr=nx=4, 1 rhs, "
                     "internal LU + last-block LU (FP64)",
         "nblock": CFG["nblock"], "n": CFG["n"], "qr": CFG["qr"], "qx": CFG["qx"],
         "nr": CFG["nr"], "nx": CFG["nx"], "nrhs": 1,
         "l2": "inputs (0.65 GB matrix) larger than L2; no flush needed"}
    if extra:
        c.update(extra)
    return c


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def replica_seeds(rank):
    """Seeds of the system and right-hand side that `rank` solves: each replica
    factors its own independent system (no data crosses ranks)."""
    return rank, 1 + rank


def max_over_ranks(dist, v, device):
    """The slowest rank's time, known to every rank (all ranks must call it in
    the same order); `dist` is None for a single process.  `device` is "cuda"
    under NCCL and "cpu" under gloo."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world, ncols, seconds):
    """Unknowns/s of the whole job: every replica solves `ncols` unknowns in
    `seconds` (the slowest rank's time)."""
    return world * ncols / seconds


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for _, _, f in rows:
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r[0] for r in rows),
                "sm_max_mhz": max(r[1] for r in rows), "reasons": sorted(reasons),
                "samples": len(rows)}


def algorithmic_bytes(d, nrhs=1):
    """Minimum HBM traffic per block (FP64): factorize reads D,E,B,C once and
    writes the factors T (2n^2), U-row D',E',B',C' once plus int32 pivots;
    solve reads the factors and reads/writes x in both sweeps."""
    n, nr, nx = d["n"], d["nr"], d["nx"]
    fact = 8 * ((2 * n * n + n * nx + nr * n) + (4 * n * n + n * nx + nr * n)) + 4 * n
    solve = 8 * (4 * n * n + n * nx + nr * n) + 4 * n + 8 * 4 * n * nrhs
    return fact * d["nblock"], solve * d["nblock"]


def launches_per_step(nblock, nr, nx):
    """Kernel launches of one factorize+solve step of the FP64 n=16 path
    (forward elimination fused into the pair kernel)."""
    def pairs(k):
        return (nblock - k - 1) // (2 * k) + 1 if nblock > k else 0
    levels, k = [], 1
    while k < nblock:
        levels.append(k)
        k *= 2
    big = [k for k in levels if pairs(k) > 16]   # one pair-kernel launch (+ border fix-up) each
    top = 1 if len(big) < len(levels) else 0     # the remaining top levels: one CTA
    fact = (1 if nr else 0) + (4 if nblock % 2 else 0) + len(big) * (2 if nr else 1) + top
    fact += (2 if nr * nx else 0) + (2 if nr else 0) + 2  # F and xb sums, assemble, last-block LU
    solve = 1 + top + len(big)                   # last-block solve, backward top, backward levels
    return fact + solve


def cpu_reference_run(s, b, steps, warmup, threads, internal="LU"):
    """The reference's own BorderedCR (oracle/_ref) on the host cores with its
    own thread pool: `warmup` untimed and `steps` timed factorize + solve runs,
    each on a fresh copy of the matrix.  Returns (times, x, the object holding
    the unfactored matrix)."""
    from oracle import pyoracle as po
    src = po.RefBCR(s, internal, "LU", "NONE", nthreads=threads, npb=threads)
    work = po.RefBCR(s, internal, "LU", "NONE", nthreads=threads, npb=threads)
    work.set_threads(True, True)
    times = []
    x = None
    for i in range(warmup + steps):
        t, x = work.time_factor_solve(src, b)
        if i >= warmup:
            times.append(t)
    return times, x, src


def accuracy(s, x, b, ref_src=None, x_ref=None):
    """Relative residual ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) with
    A x from the reference's own Mv (ref_src, an unfactored RefBCR; the C
    oracle's Mv when the reference is not built) and the forward error
    ||x - x_ref||_inf / ||x_ref||_inf against the reference solution.  x, b
    may hold several right-hand sides (rows); the worst column is reported."""
    from oracle import pyoracle as po
    mv = ref_src.mv if ref_src is not None else po.Oracle(s).mv
    X = np.atleast_2d(x)
    Bm = np.atleast_2d(b)
    nA = s.norm_inf()
    rel = 0.0
    for c in range(X.shape[0]):
        r = Bm[c, :s.nrows] - mv(X[c, :s.ncols])
        rel = max(rel, float(np.abs(r).max() / (nA * np.abs(X[c, :s.ncols]).max() + np.abs(Bm[c, :s.nrows]).max())))
    out = {"rel_residual": rel, "residual_mv": "reference" if ref_src is not None else "oracle"}
    if x_ref is not None:
        XR = np.atleast_2d(x_ref)
        fe = max(float(np.abs(X[c, :s.ncols] - XR[c, :s.ncols]).max() / np.abs(XR[c, :s.ncols]).max())
                 for c in range(X.shape[0]))
        out["fwd_err"] = fe
        out["fwd_err_vs"] = "reference BorderedCR (oracle/_ref)"
    return out


def reference_point(s, b, threads, internal="LU", runs=1):
    """The reference BorderedCR's time and solution for system s (None when
    oracle/_ref is not built)."""
    from oracle import pyoracle as po
    if not po.ref_available():
        return None
    times, x, src = cpu_reference_run(s, b, runs, 0, threads, internal)
    t = statistics.median(times)
    return {"t": t, "x": x, "src": src,
            "json": {"ms": t * 1e3, "value": s.ncols / t, "unit": "unknowns/s", "cores": threads,
                     "kind": "reference", "runs": runs}}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from alglin_b200 import synth
    from oracle import pyoracle as po
    if not po.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libbcr_ref.so was not built"}))
        return 0
    s = synth.collocation(**CFG, seed=0)
    b = synth.rhs(s, 1, seed=1)[0]
    threads = os.cpu_count() or 1
    steps, warm = args.steps, args.warmup
    times, x, src = cpu_reference_run(s, b, steps, warm, threads)
    t = statistics.median(times)
    v = s.ncols / t
    line = {"metric": METRIC, "value": v, "unit": "unknowns/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": warm, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": workload_config(), "cpu_threads": threads,
            "cpu_baseline": {"value": v, "unit": "unknowns/s", "cores": threads, "kind": "reference",
                             "sample": "full workload, median of %d factorize+solve runs after %d "
                                       "untimed" % (steps, warm)},
            "e2e": {"value": v, "unit": "unknowns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    line.update(accuracy(s, x, b, src))
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA GPU")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from alglin_b200 import bcr, synth

    seed_s, seed_b = replica_seeds(rank)
    s = synth.collocation(**CFG, seed=seed_s)
    b = synth.rhs(s, 1, seed=seed_b)[0]
    L = max(s.nrows, s.ncols)
    h = bcr.BorderedCR()
    h.load_system(s)
    h.select("LU")
    h.select_last("LU")
    h.upload()
    b_dev = torch.from_numpy(b).cuda()
    x_dev = torch.empty_like(b_dev)
    torch.cuda.synchronize()
    # The step (factorize + copy of the rhs + solve) is replayed as a CUDA graph
    # on the handle's own stream; the factorization status is read once after
    # the timed region.
    stream = torch.cuda.ExternalStream(h.stream())
    h.graph_capture(bcr.GRAPH_FACTORIZE)
    h.graph_capture(bcr.GRAPH_SOLVE, 1, x_dev.data_ptr(), L, b_dev.data_ptr())
    h.graph_capture(bcr.GRAPH_STEP, 1, x_dev.data_ptr(), L, b_dev.data_ptr())
    for _ in range(args.warmup):
        h.graph_launch(bcr.GRAPH_STEP)
    h.synchronize()
    assert h.factorize_status(), h.last_error()

    def timed(what, reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            h.graph_launch(what)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    fact_ms = timed(bcr.GRAPH_FACTORIZE, args.steps)
    solve_ms = timed(bcr.GRAPH_SOLVE, args.steps)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms = timed(bcr.GRAPH_STEP, args.steps)
    clocks = clk.summary()
    assert h.factorize_status(), h.last_error()
    ms = max_over_ranks(dist, ms, "cuda")
    value = whole_job_value(world, s.ncols, ms * 1e-3)
    x = x_dev.cpu().numpy()

    if args.no_e2e:
        acc = accuracy(s, x, b)
        print(json.dumps({"value": value, "ms_per_step": ms, "phases_ms": {"factorize": fact_ms, "solve": solve_ms},
                          "nblock": CFG["nblock"], "clocks": clocks, **acc}))
        return 0
    # end to end through the C ABI with host buffers: factorize + solve in one
    # call; every step uploads the matrix from the handle's page-locked host
    # copy and the right-hand side from a page-locked buffer, into which the
    # solution comes back
    xh = torch.empty(b.shape, dtype=torch.float64, pin_memory=True).numpy()
    xh[:] = b
    for _ in range(2):
        assert h.factorize_solve(1, xh, L), h.last_error()
        xh[:] = b
    nbytes_mat = sum(getattr(s, k).nbytes for k in ("D", "E", "B", "C", "Cq", "F", "H"))
    te = []
    for _ in range(max(3, min(args.steps, 10))):
        xh[:] = b
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        assert h.factorize_solve(1, xh, L), h.last_error()
        te.append(time.perf_counter() - t0)
    e2e_t = max_over_ranks(dist, statistics.median(te), "cuda")

    fact_b, solve_b = algorithmic_bytes(CFG)
    peak, peak_kind = load_peaks()
    achieved = fact_b / (fact_ms * 1e-3) / 1e9
    line = None
    if rank == 0:
        cpu, ref = None, None
        if world == 1 and not args.no_cpu:
            cpu, ref = cpu_baseline(s, b, args.steps, args.warmup)
        line = {
            "metric": METRIC, "value": value, "unit": "unknowns/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "ours",
            "config": workload_config(), "parallelism": f"replicas x{world}",
            "phases_ms": {"factorize": fact_ms, "solve": solve_ms},
            "roofline": {"bound": "hbm", "kernel": "factorize (every CR level launch, the top-level CTA, "
                                                   "the F/xb sums and the last block)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": FACT_DRAM_BYTES_PER_BLOCK * CFG["nblock"],
                         "traffic_source": "ncu dram__bytes_read+write of one factorization of this "
                                           "workload at nblock=40000, 21,542 B per block, scaled to "
                                           "100000 blocks (profiles/dram_factor_solve_n16_nblock40000.md)",
                         "algorithmic_bytes": fact_b},
            "e2e": {"value": whole_job_value(world, s.ncols, e2e_t), "unit": "unknowns/s",
                    "h2d_bytes_per_step": nbytes_mat + 8 * L, "d2h_bytes_per_step": 8 * L},
            "gpu_launches": launches_per_step(CFG["nblock"], CFG["nr"], CFG["nx"]) * args.steps,
            "clocks": clocks,
        }
        line.update(accuracy(s, x, b, ref["src"] if ref else None, ref["x"] if ref else None))
        if cpu:
            line["cpu_baseline"] = cpu
        if not args.no_variants and world == 1:
            threads = os.cpu_count() or 1
            line["variants"] = variants(torch, bcr, synth, min(args.steps, 10), 3, rank, threads,
                                        s, b, ref, h)
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def graph_step_time(torch, bcr, h, s, b, steps, warmup, prec, nrhs=1):
    """Device time of one factorize + solve graph step of system s on handle h
    (b: one right-hand side, or nrhs of them as rows).  Returns the timing
    entry and the solution."""
    L = max(s.nrows, s.ncols)
    h.set_precision(prec)
    h.upload()
    bb = np.ascontiguousarray(np.atleast_2d(b)[:, :L])
    b_dev = torch.from_numpy(bb).cuda()
    x_dev = torch.empty_like(b_dev)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(h.stream())
    h.graph_capture(bcr.GRAPH_STEP, nrhs, x_dev.data_ptr(), L, b_dev.data_ptr())
    for _ in range(warmup):
        h.graph_launch(bcr.GRAPH_STEP)
    h.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        h.graph_launch(bcr.GRAPH_STEP)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    assert h.factorize_status(), h.last_error()
    it, rr = h.refinement_info()
    x = x_dev.cpu().numpy()
    return {"value": s.ncols / (ms * 1e-3), "unit": "unknowns/s", "ms_per_step": ms,
            "refinement_steps": it if prec else 0}, (x if nrhs > 1 else x[0])


def _entry(timing, s, x, b, ref, **extra):
    e = dict(timing)
    e.update(accuracy(s, x, b, ref["src"] if ref else None, ref["x"] if ref else None))
    if ref:
        e["reference"] = ref["json"]
    e.update(extra)
    return e


def variants(torch, bcr, synth, steps, warmup, rank, threads, sB, bB, refB, hB):
    """The other measured paths (see the module docstring), each with its
    residual and forward error against the reference BorderedCR's solution of
    the same system and the reference's time on the host cores."""
    from oracle import pyoracle as po
    out = {}
    # n=8 nblock=1000: the reference's CPU-runnable case
    cA = dict(synth.CONFIGS["A"])
    sA = synth.collocation(**cA, seed=rank)
    bA = synth.rhs(sA, 1, seed=1 + rank)[0]
    hA = bcr.BorderedCR()
    hA.load_system(sA)
    tA, xA = graph_step_time(torch, bcr, hA, sA, bA, steps, warmup, bcr.PRECISION_FP64)
    refA = reference_point(sA, bA, threads, runs=5)
    out["A_fp64"] = _entry(tA, sA, xA, bA, refA, workload="trapezoid-collocation BABD n=8 nblock=1000 nr=nx=2, 1 rhs")
    del hA
    wlB = "trapezoid-collocation BABD n=16 nblock=100000 qr=qx=2 nr=nx=4"
    # mixed path on the headline system
    hB.select("LU")
    t, x = graph_step_time(torch, bcr, hB, sB, bB, steps, warmup, bcr.PRECISION_MIXED)
    out["B_mixed"] = _entry(t, sB, x, bB, refB, workload=wlB + ", 1 rhs")
    # 8 right-hand sides: factorize + solve(8, ...)
    b8 = synth.rhs(sB, 8, seed=11 + rank)
    t, x8 = graph_step_time(torch, bcr, hB, sB, b8, steps, warmup, bcr.PRECISION_FP64, nrhs=8)
    ref8 = None
    if refB:
        tt, xr8, _ = cpu_reference_run(sB, b8, 1, 0, threads)
        ref8 = {"x": xr8, "src": refB["src"],
                "json": {"ms": tt[0] * 1e3, "value": sB.ncols / tt[0], "unit": "unknowns/s", "cores": threads,
                         "kind": "reference", "runs": 1}}
    t["solutions_per_s"] = 8 * 1e3 / t["ms_per_step"]
    out["B_fp64_rhs8"] = _entry(t, sB, x8, b8, ref8, workload=wlB + ", factorize + solve(8, X, ld)")
    # QR panels
    hB.select("QR")
    t, x = graph_step_time(torch, bcr, hB, sB, bB, steps, warmup, bcr.PRECISION_FP64)
    refQ = reference_point(sB, bB, threads, internal="QR")
    out["B_fp64_QR"] = _entry(t, sB, x, bB, refQ, workload=wlB + ", internal QR, 1 rhs")
    hB.select("LU")
    del refQ
    # the reference's own BorderedCR<float> (no refinement) on the host cores
    if po.ref_available():
        tf, xf = po.ref_f32_factor_solve(sB, bB, threads, threads)
        out["B_reference_f32_cpu"] = _entry({"value": sB.ncols / tf, "unit": "unknowns/s", "ms_per_step": tf * 1e3,
                                             "cores": threads}, sB, xf, bB, refB,
                                            workload=wlB + ", reference BorderedCR<float> on the host cores, "
                                                           "unrefined FP32")
    # n=32 nblock=65536 at three condition levels
    cC = dict(synth.CONFIGS["C"])
    for kappa in (1.0, 10.0, 100.0):
        sC = synth.collocation(**cC, kappa=kappa, seed=rank)
        bC = synth.rhs(sC, 1, seed=1 + rank)[0]
        hC = bcr.BorderedCR()
        hC.load_system(sC)
        refC = reference_point(sC, bC, threads)
        f64, x64 = graph_step_time(torch, bcr, hC, sC, bC, steps, warmup, bcr.PRECISION_FP64)
        mix, xmx = graph_step_time(torch, bcr, hC, sC, bC, steps, warmup, bcr.PRECISION_MIXED)
        wl = "trapezoid-collocation BABD n=32 nblock=65536 nr=nx=8 kappa=%g, 1 rhs" % kappa
        k = "%g" % kappa
        out["C_fp64_k" + k] = _entry(f64, sC, x64, bC, refC, workload=wl)
        out["C_mixed_k" + k] = _entry(mix, sC, xmx, bC, refC, workload=wl)
        out["C_mixed_over_fp64_k" + k] = mix["value"] / f64["value"]
        del hC, sC, refC
    # n=128 nblock=8192: tcgen05 split-precision pair kernel on the mixed path
    cE = dict(synth.CONFIGS["E"])
    sE = synth.collocation(**cE, seed=rank)
    bE = synth.rhs(sE, 1, seed=1 + rank)[0]
    hE = bcr.BorderedCR()
    hE.load_system(sE)
    f64, x64 = graph_step_time(torch, bcr, hE, sE, bE, steps, warmup, bcr.PRECISION_FP64)
    mix, xmx = graph_step_time(torch, bcr, hE, sE, bE, steps, warmup, bcr.PRECISION_MIXED)
    del hE
    refE = reference_point(sE, bE, threads)
    wl = "trapezoid-collocation BABD n=128 nblock=8192 qr=qx=4 nr=nx=16, 1 rhs"
    out["E_fp64"] = _entry(f64, sE, x64, bE, refE, workload=wl, pair_kernel="FP64 blocked LU, DMMA products")
    out["E_mixed"] = _entry(mix, sE, xmx, bE, refE, workload=wl, pair_kernel="FP32 LU, tcgen05 3xTF32 products")
    out["E_mixed_over_fp64"] = mix["value"] / f64["value"]
    del sE, refE
    for name, prec, sched, ref in (("D_batched_fp64", bcr.PRECISION_FP64, bcr.BATCH_LEVELS, True),
                                   ("D_batched_mixed", bcr.PRECISION_MIXED, bcr.BATCH_LEVELS, True),
                                   ("D_batched_fp64_persistent", bcr.PRECISION_FP64, bcr.BATCH_PERSISTENT, False)):
        try:
            out[name] = batched(torch, bcr, synth, rank, prec, threads, schedule=sched, reference=ref)
        except Exception as e:  # e.g. not enough device memory on a shared GPU
            out[name] = {"unavailable": str(e)[:200]}
        torch.cuda.empty_cache()
    return out


def batched(torch, bcr, synth, rank, prec, threads, nsys=4096, sample_every=32, schedule=None, reference=True):
    """4096 independent systems, nblock ~ U{64..4096}, n in {4,8,16,32},
    nr = nx in {0,2,4}: one CUDA graph per factorize + solve of the whole batch.
    Every 32nd system (128 in all) is also copied to the host: its GPU solution
    is checked against the reference BorderedCR (residual with the reference's
    Mv, forward error), and the reference solves those 128 systems with one
    BorderedCR object per system (npb = 1) spread over the host cores, which
    gives the reference's systems/s on the same mix."""
    from concurrent.futures import ThreadPoolExecutor

    from cuda.bindings import runtime as rt
    from oracle import pyoracle as po
    dims = synth.batch_dims(nsys, 64, 4096, seed=rank)
    bt = bcr.Batch()
    for d in dims:
        bt.add_device(*d)
    bt.set_precision(prec)
    bt.set_schedule(bcr.BATCH_LEVELS if schedule is None else schedule)
    bt.prepare()
    g = torch.Generator(device="cuda")
    g.manual_seed(7 + rank)
    kept = {}
    for i, d in enumerate(dims):
        ts = synth.collocation_torch(torch, *d, seed=i + nsys * rank)
        r, c = bt.system_size(i)
        rhs = torch.zeros(max(r, c), dtype=torch.float64, device="cuda")
        rhs[:r] = torch.randn(r, generator=g, device="cuda", dtype=torch.float64)
        torch.cuda.synchronize()  # the blocks and rhs are complete before they are copied
        bt.load_device(i, *[t.data_ptr() if t.numel() else 0 for t in ts])
        rt.cudaMemcpy(bt.device_b(i), rhs.data_ptr(), max(r, c) * 8, rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
        if i % sample_every == 0:
            arr = [t.cpu().numpy() for t in ts]
            kept[i] = (synth.BABD(*d, D=arr[0], E=arr[1], B=arr[2], C=arr[3], Cq=arr[4], F=arr[5], H=arr[6]),
                       rhs.cpu().numpy())
    bt.autotune()
    bt.graph_capture()
    stream = torch.cuda.ExternalStream(bt.stream())
    for _ in range(3):
        bt.graph_launch()
    bt.synchronize()
    lat = []
    for _ in range(10):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bt.graph_launch()
        e1.record(stream)
        e1.synchronize()
        lat.append(e0.elapsed_time(e1))
    ok = bt.check_status()
    iters, worst = bt.refinement_info()
    lat.sort()
    p50, p99 = lat[len(lat) // 2], lat[-1]
    unk = sum(n * (nb + 1) + nx for nb, n, _, _, _, nx in dims)
    out = {"systems_per_s": nsys / (p50 * 1e-3), "unknowns_per_s": unk / (p50 * 1e-3),
           "p50_ms": p50, "p99_ms": p99, "nsys": nsys, "all_factorized": bool(ok),
           "refinement_steps": iters, "worst_rel_residual_device": worst if prec else None,
           "classes": [{"n": c[0], "systems": c[1], "family": ["auto", "tc", "grp", "rows"][c[2]],
                        "pairs_per_cta": c[3]} for c in bt.classes()],
           "workload": "4096 systems, nblock U{64..4096}, n in {4,8,16,32}, nr=nx in {0,2,4}, "
                       "collocation blocks drawn on the device"}
    # the sampled systems' solutions, checked against the reference
    xs = {}
    for i, (s, _) in kept.items():
        xh = np.zeros(max(s.nrows, s.ncols))
        rt.cudaMemcpy(xh.ctypes.data, bt.device_x(i), xh.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        xs[i] = xh
    out["schedule"] = "persistent (one launch per class, per-system level schedule)" \
        if schedule == bcr.BATCH_PERSISTENT else "one launch per level"
    if reference and po.ref_available():
        def ref_one(i):
            s, rhs = kept[i]
            src = po.RefBCR(s, "LU", "LU", "NONE", nthreads=0)
            work = po.RefBCR(s, "LU", "LU", "NONE", nthreads=0)
            t, xr = work.time_factor_solve(src, rhs)
            return i, t, xr, src
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=threads) as ex:
            res = list(ex.map(ref_one, sorted(kept)))
        wall = time.perf_counter() - t0
        worst_r, worst_f = 0.0, 0.0
        for i, t, xr, src in res:
            s, rhs = kept[i]
            a = accuracy(s, xs[i], rhs, src, xr)
            worst_r = max(worst_r, a["rel_residual"])
            worst_f = max(worst_f, a["fwd_err"])
        out["rel_residual"] = worst_r
        out["fwd_err"] = worst_f
        out["accuracy_sample"] = "%d systems (every %dth), worst over the sample, reference Mv and solution" % (
            len(kept), sample_every)
        out["reference"] = {"systems_per_s": len(kept) / wall, "cores": threads, "kind": "reference",
                            "sample": "the same %d systems, one BorderedCR object per system (npb=1) on a "
                                      "pool of %d host threads, factorize + solve" % (len(kept), threads)}
    return out


def cpu_baseline(s, b, steps, warmup):
    """The reference arm's measurement, run inside this arm: the reference
    BorderedCR on the host cores, `warmup` untimed then `steps` timed
    factorize + solve runs (median).  Returns (cpu_baseline entry, reference
    point with the solution)."""
    from oracle import pyoracle as po
    threads = os.cpu_count() or 1
    if po.ref_available():
        times, x, src = cpu_reference_run(s, b, steps, warmup, threads)
        t = statistics.median(times)
        return ({"value": s.ncols / t, "unit": "unknowns/s", "cores": threads, "kind": "reference",
                 "sample": "full workload, median of %d factorize+solve runs after %d untimed, reference "
                           "BorderedCR with its own thread pool" % (steps, warmup)},
                {"x": x, "src": src, "json": {"ms": t * 1e3, "value": s.ncols / t, "cores": threads}})
    o = po.Oracle(s, "LU", "LU")
    t0 = time.perf_counter()
    o.factorize()
    o.solve(b)
    t = time.perf_counter() - t0
    return ({"value": s.ncols / t, "unit": "unknowns/s", "cores": 1, "kind": "port",
             "sample": "full workload, one factorize+solve of the C oracle"}, None)


def run_once_batch(args):
    """One factorize + solve of a batch of --nsys-once uneven systems (the
    batch workload's systems, right-hand sides of ones) with the default
    per-level schedule, for profilers."""
    import torch
    from alglin_b200 import bcr, synth
    dims = synth.batch_dims(args.nsys_once, 64, 4096, seed=0)
    bt = bcr.Batch()
    for d in dims:
        bt.add_device(*d)
    bt.set_precision(bcr.PRECISION_MIXED if args.precision == "mixed" else bcr.PRECISION_FP64)
    bt.prepare()
    for i, d in enumerate(dims):
        ts = synth.collocation_torch(torch, *d, seed=i)
        torch.cuda.synchronize()
        bt.load_device(i, *[t.data_ptr() if t.numel() else 0 for t in ts])
    xs = [np.ones(max(bt.system_size(i))) for i in range(len(dims))]
    assert bt.factorize_solve(xs), bt.last_error()
    print(json.dumps({"once": "D", "nsys": len(dims), "precision": args.precision,
                      "classes": bt.classes(), "refinement": bt.refinement_info()}))
    return 0


def run_once(args):
    """One factorize + solve of a named workload through the C ABI, for profilers."""
    import torch
    from alglin_b200 import bcr, synth
    if args.once == "D":
        return run_once_batch(args)
    cfg = dict(synth.CONFIGS[args.once])
    if args.nblock_once:
        cfg["nblock"] = args.nblock_once
    s = synth.collocation(**cfg, seed=0)
    b = synth.rhs(s, 1, seed=1)[0]
    L = max(s.nrows, s.ncols)
    h = bcr.BorderedCR()
    h.load_system(s)
    h.set_precision(bcr.PRECISION_MIXED if args.precision == "mixed" else bcr.PRECISION_FP64)
    h.upload()
    x = torch.from_numpy(b).cuda()
    torch.cuda.synchronize()
    h.factorize_solve_device(1, x.data_ptr(), L)
    h.synchronize()
    assert h.factorize_status(), h.last_error()
    print(json.dumps({"once": args.once, "nblock": cfg["nblock"], "precision": args.precision,
                      "refinement": h.refinement_info()}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the mixed-path, n=32 and batched measurements")
    ap.add_argument("--nblock", type=int, default=CFG["nblock"],
                    help="smaller systems for profiling runs (the reported workload is 100000)")
    ap.add_argument("--nsys-once", type=int, default=64, help="systems of the --once D batch")
    ap.add_argument("--once", choices=["A", "B", "C", "D", "E"],
                    help="run one factorize+solve of that workload and exit (for profilers)")
    ap.add_argument("--nblock-once", type=int, default=0, help="nblock of the --once workload")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"], help="path of --once")
    args = ap.parse_args()
    if args.once:
        return run_once(args)
    CFG["nblock"] = args.nblock
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
