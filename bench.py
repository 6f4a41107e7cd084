#!/usr/bin/env python
"""Benchmark: batched interior-point solves per second on B200.

Workload (one "step"): one batch of synthetic portfolio QP/SOCP instances solved to the 1e-8 gap
(4096 per GPU by default: n_assets ~ U[50, 400], factor model F (n x 10), D ~ U(0.1, 1), budget
equality, long-only cone, SOC risk bound), all instances in one persistent launch.  Both factor
precisions are timed (FP64 and mixed FP32/FP64), with per-instance p50/p99 latency from the
device's global timer.

  value  — solves/s with every input resident in HBM (device time, CUDA events on the launching
           stream, max over ranks)
  e2e    — solves/s through the public C ABI (mb_batch_solve) from host problems to host results:
           symbolic analysis, packing, H2D, solve and D2H inside the timed region (wall clock)

Multi-GPU: one process per GPU, each solving its own batch (independent instances; no collective
on the data path; weak scaling).  `--impl reference` times the reference algorithm's CPU
restatement (the FP64 oracle) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mumblebee.jl_b200"))

import numpy as np  # noqa: E402

WORKLOAD = ("batched portfolio QP/SOCP: n_assets~U[50,400], F n x 10 N(0,1), D~U(0.1,1), "
            "budget equality, long-only cone, SOC risk bound; solve to 1e-8 gap")
METRIC = "IPM solves/s & p50/p99 latency at 1e-8 gap: mixed vs FP64 GPU; factor TC%"
# DRAM bytes (read + write) of one ipm_batch_kernel launch per instance of this workload, FP64
# factor: an ncu capture of a smaller launch of the same instance distribution, divided by its
# instance count (profiles/ipm_batch_kernel_portfolio_fp64.txt gives the command and the figures)
TRAFFIC_BYTES_PER_INSTANCE_FP64 = 82.35e9 / 296
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one 296-instance launch (82.35 GB), "
                  "scaled to this launch by instance count")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--count", type=int, default=4096, help="instances per step per GPU")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "mixed"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--ref-per-core", type=int, default=8, help="reference arm: instances per host core per step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the other precision's arm")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving arm")
    ap.add_argument("--no-tune", action="store_true", help="launch configuration without the autotuner")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="offered requests per second")
    ap.add_argument("--serve-seconds", type=float, default=1.0, help="length of the arrival window")
    ap.add_argument("--serve-nmin", type=int, default=100)
    ap.add_argument("--serve-nmax", type=int, default=2000)
    ap.add_argument("--serve-arena-gb", type=int, default=32)
    ap.add_argument("--extras", default="", choices=["", "stable", "comp", "coop", "config4", "all"],
                    help="instead of the main line: one JSON line each for the stable factor against the default "
                         "one, the compensated products, one grid-cooperative SOCP solve (n = 2000), and the "
                         "n = 20000 exponential/power-cone problem (1 GPU; 'all' runs the first three)")
    ap.add_argument("--config4-scale", type=float, default=1.0,
                    help="size of the exponential/power-cone problem relative to n = 20000")
    ap.add_argument("--fp32-tiles", type=int, default=0, choices=[0, 1, 2],
                    help="settings.fp32_tiles of every arm: 0 the runtime's choice, 1 FFMA, 2 tensor cores")
    ap.add_argument("--extras-count", type=int, default=1184, help="instances of the stable-factor arm")
    ap.add_argument("--comp-rows", type=int, default=1 << 20, help="rows = columns of the compensated-product matrix")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------ dist
def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return ws, rank, local, pg


def allreduce_max(pg, x, local):
    if pg is None:
        return x
    import torch
    dev = f"cuda:{local}" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, local):
    if pg is not None:
        import torch
        if torch.cuda.is_available():
            pg.barrier(device_ids=[local])
        else:
            pg.barrier()


# ------------------------------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, local):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-i",
                                       str(local), "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush(); self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1])); mx.append(float(c[2]))
            except ValueError:
                continue
            for nm, v in zip(names, c[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------------ peaks
def measure_peaks():
    """FP64 and TF32 dense GEMM peaks measured live (torch/cuBLAS, 8192^3, best of 5): the
    denominators of the factorization roofline (MEASURED_PEAKS.json carries HBM and BF16 only)."""
    import torch
    out = {}
    n = 8192
    for name, dt, tf32 in (("fp64", torch.float64, False), ("tf32", torch.float32, True)):
        torch.backends.cuda.matmul.allow_tf32 = tf32
        a = torch.randn(n, n, device="cuda", dtype=dt)
        b = torch.randn(n, n, device="cuda", dtype=dt)
        for _ in range(2):
            a @ b
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(); a @ b; e1.record(); torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        out[name] = 2 * n ** 3 / best / 1e12
        del a, b
    torch.backends.cuda.matmul.allow_tf32 = False
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------------------------------------ oracle
# ------------------------------------------------------------------------------------------ main
def make_problems(count, seed, rank, ctx):
    from mumblebee_b200 import generators as G
    from mumblebee_b200.ipm import IPMProblem, PositiveCone, CofreeCone, SecondOrderCone
    rng = np.random.default_rng([seed, rank])
    sizes = rng.integers(50, 401, size=count)
    cones = {0: CofreeCone(), 1: PositiveCone(), 2: SecondOrderCone()}
    probs = []
    for i, n in enumerate(sizes):
        pb = G.portfolio(int(n), rng=np.random.default_rng([seed, rank, i]))
        probs.append(IPMProblem(pb["Q"], pb["B"], pb["f"], pb["g"], pb["mu"], [cones[k] for k in pb["kinds"]],
                                pb["sizes"], ctx=ctx))
    return probs, sizes


_REF_PROBS = None


def _ref_init(seed, idx):
    """Pool initializer of the reference arm: build the oracle's block form of instances `idx` of
    the GPU arm's own seeded list (make_problems' sizes and per-instance seeds, rank 0) with the
    oracle's ordering, once per worker, outside the timed region."""
    global _REF_PROBS
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import frontend
    import oracle
    from mumblebee_b200 import generators as G
    oracle.lib(threads=1)
    sizes = np.random.default_rng([seed, 0]).integers(50, 401, size=max(idx) + 1)
    _REF_PROBS = {}
    for i in idx:
        pb = G.portfolio(int(sizes[i]), rng=np.random.default_rng([seed, 0, i]))
        prob = frontend.ipmproblem_from_csc(pb["Q"], pb["B"], pb["f"], pb["g"], pb["mu"], pb["kinds"], pb["sizes"],
                                            pb["params"])
        adj, w = frontend.vertex_graph(prob)
        _REF_PROBS[i] = (prob, frontend.minimum_degree(adj, w))


def _ref_solve(i):
    import oracle
    prob, vp = _REF_PROBS[i]
    r = oracle.OracleSolver(prob, oracle.default_settings(), vperm=vp, threads=1).solve()
    return i, r["status"], r["niter"]


def oracle_steps(args, steps, warmup):
    """The reference algorithm's FP64 CPU restatement (the oracle; the reference itself is a Julia
    package and Julia is absent) on every host core.  One step solves the first K instances of the
    GPU arm's own list (same sizes and seeds), largest first, one instance per process at a time;
    K = ref_per_core per core, so that a step is a bounded sample of the workload.  Timed by the
    host clock around each step (problem construction excluded, as for the GPU)."""
    cores = os.cpu_count() or 1
    k = min(args.count, args.ref_per_core * cores)
    sizes = np.random.default_rng([args.seed, 0]).integers(50, 401, size=k)
    order = [int(i) for i in np.argsort(-sizes, kind="stable")]
    ctx = mp.get_context("spawn")
    ms, status = [], []
    with ctx.Pool(cores, initializer=_ref_init, initargs=(args.seed, list(range(k)))) as pool:
        for _ in range(warmup):
            pool.map(_ref_solve, order, chunksize=1)
        for _ in range(steps):
            t = time.perf_counter()
            status = pool.map(_ref_solve, order, chunksize=1)
            ms.append(1e3 * (time.perf_counter() - t))
    opt = sum(1 for _, st, _ in status if st == "OPTIMAL")
    sample = (f"instances 0..{k - 1} of the {args.count}-instance list (same sizes and seeds) per step, FP64 oracle "
              f"(CPU restatement of the reference; Julia is not installed), {cores} processes x 1 OpenBLAS thread, "
              f"largest first; {opt}/{k} OPTIMAL")
    return k, ms, cores, sample


def run_reference(args, ws, rank):
    """`--impl reference`: rank 0 alone times the oracle steps; other ranks exit without work."""
    if rank != 0:
        return
    k, ms, cores, sample = oracle_steps(args, args.steps, args.warmup)
    step_ms = statistics.mean(ms)
    v = k / (step_ms / 1e3)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "step_ms": ms,
            "instances_per_step": k, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": main_config(args, ws),
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main_config(args, ws):
    """The workload's name and sizes, identical in both arms."""
    return {"workload": WORKLOAD, "instances_per_gpu": args.count, "precision": args.precision,
            "parallelism": f"instances sharded over {ws} GPU(s), one persistent launch per step",
            "l2": "inputs and workspace larger than the 126 MB L2 (sizes under footprint)"}


def timed_arm(probs, precision, args, pg, local, ws, ctx, lower):
    """Prepare a batch at `precision`, warm up, time `steps` persistent launches (CUDA events on the
    launching stream, max over ranks) and read back statuses, iterations and latencies.  The launch
    configuration (kernel build and resident instances per SM) is the autotuner's choice from
    timed trial launches on a sample of the same instances, unless --fp32-tiles fixes the build."""
    from mumblebee_b200.autotune import tune
    from mumblebee_b200.ipm import Batch, IPMSettings
    settings = IPMSettings(precision=precision, fp32_tiles=args.fp32_tiles)
    t0 = time.time()
    tuned = None
    grid = 0
    if args.fp32_tiles == 0 and not args.no_tune:
        import torch
        nsm = torch.cuda.get_device_properties(local).multi_processor_count
        choice = tune(probs, settings, nsm=nsm, seed=args.seed)
        settings, grid = choice.settings, choice.grid
        tuned = dict(choice.as_dict(), tune_s=round(time.time() - t0, 2))
    t0 = time.time()
    batch = Batch(probs, settings, ctx=ctx)
    t_prep = time.time() - t0
    st = batch.stats()
    for _ in range(args.warmup):
        batch.run(grid=grid)
    barrier(pg, local)
    clk = Clocks(local)
    ms_steps = [batch.run(grid=grid) for _ in range(args.steps)]
    clocks = clk.stop()
    ms = sum(ms_steps) / len(ms_steps)
    ms_max = allreduce_max(pg, ms, local)
    res = batch.fetch(want_vectors=False)          # results of the last timed launch
    lat, svc = batch.latencies_ms()
    tm = batch.timers()
    ntrsv = tm[:, batch.SECTIONS.index("ntrsv")]
    # section clocks of the largest quarter of the instances (by n), mean per instance, Mclk
    nsz = np.array([z["n"] for z in batch.sizes])
    big = nsz >= np.percentile(nsz, 75)
    sections = {k: round(float(tm[big, j].mean()) / (1e6 if not k.startswith("n") else 1.0), 2)
                for j, k in enumerate(batch.SECTIONS)}
    sections["instances"] = int(big.sum())
    sections["iters_mean"] = float(np.mean([r.niter for r, b in zip(res, big) if b]))
    out = {"precision": precision, "autotune": tuned, "settings": settings, "grid": grid, "sections_mclk": sections, "ms": ms, "ms_max": ms_max, "ms_steps": ms_steps, "clocks": clocks,
           "value": args.count * ws / (ms_max / 1e3), "res": res, "stats": st, "prepare_s": t_prep,
           "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max())},
           "solve_ms": {"p50": float(np.percentile(svc, 50)), "p99": float(np.percentile(svc, 99))},
           "optimal": sum(1 for r in res if r.status.name == "OPTIMAL"),
           "near_optimal": sum(1 for r in res if r.status.name == "NEAR_OPTIMAL"),
           "iters_mean": float(np.mean([r.niter for r in res])),
           "flops": float(sum(r.nfactor * r.factor_flops for r in res))}
    out.update(factor_accounting(res, ntrsv, lower, precision))
    del batch
    return out


def lower_entries(probs):
    """Stored lower-triangle entries of each instance's factor: Σ over fronts of r (r + 1) / 2, r the
    front's order (residual + separator columns), from the host symbolic analysis."""
    out = []
    for p in probs:
        s = p.symbolic()
        r = (np.asarray(s["nres"]) + np.asarray(s["nsep"])).astype(np.float64)
        out.append(float((r * (r + 1) / 2).sum()))
    return np.array(out)


def factor_accounting(res, ntrsv, lower, precision):
    """Factorizations by precision and the launch's algorithmic DRAM bytes.  In the mixed path every
    iteration factors in FP32 first; an iteration redone in FP64 (nfallback) adds an FP64
    factorization, and after the switch every factorization is FP64, so the FP32 count is
    nfp32 + nfallback (capped by nfactor) and the rest are FP64.  Algorithmic bytes: a
    factorization reads the assembled BᵀB (8 B per lower entry) and writes L once (8 B FP64, 4 B FP32);
    a triangular-solve sweep reads L once."""
    n32 = np.array([min(r.nfactor, r.nfp32 + r.nfallback) if precision != "fp64" else 0 for r in res], float)
    if precision == "fp32":
        n32 = np.array([r.nfactor for r in res], float)
    nfac = np.array([r.nfactor for r in res], float)
    n64 = nfac - n32
    ff = np.array([r.factor_flops for r in res])
    # a sweep reads the factor of its iteration: FP32 on the FP32 share of the factorizations
    esz = 8.0 - 4.0 * n32 / np.maximum(nfac, 1.0)
    alg = float((n64 * 16 * lower + n32 * 12 * lower + ntrsv * esz * lower).sum())
    return {"flops_fp32": float((n32 * ff).sum()), "flops_fp64": float((n64 * ff).sum()),
            "factorizations": {"fp32": float(n32.sum()), "fp64": float(n64.sum())}, "alg_bytes": alg,
            "trsv_sweeps": float(np.sum(ntrsv))}


def serve_arm(args, ctx):
    """Serving workload: distinct requests from the seeded SOCP / portfolio QP / max-cut SDP mix
    (target n log-uniform in [serve_nmin, serve_nmax]) submitted to the continuous-batching server
    on a Poisson schedule at the offered rate.  Latency = results ready − submitted, on the server's
    host clock; solves/s = completed ÷ (last finish − first submit)."""
    from mumblebee_b200 import generators as G
    from mumblebee_b200.ipm import IPMProblem, IPMSettings, Server, _CONES
    nreq = max(1, int(args.serve_rate * args.serve_seconds))
    mix = G.serving_mix(nreq + 6, seed=args.seed + 7, nmin=args.serve_nmin, nmax=args.serve_nmax)
    probs = [IPMProblem(pb["Q"], pb["B"], pb["f"], pb["g"], pb["mu"], [_CONES[k]() for k in pb["kinds"]],
                        pb["sizes"], ctx=ctx) for _, pb in mix]
    kinds = [k for k, _ in mix]
    srv = Server(IPMSettings(precision=args.precision), arena_bytes=args.serve_arena_gb << 30, capacity=8192,
                 planners=os.cpu_count() or 1, ctx=ctx)
    for t in [srv.submit(p) for p in probs[nreq:]]:      # warm-up: module load, first launch
        srv.wait(t, 600.0)
        srv.result(t)
    rng = np.random.default_rng(args.seed + 11)
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, nreq))
    t0 = time.perf_counter()
    tickets = []
    for i in range(nreq):
        while True:
            dt = arrivals[i] - (time.perf_counter() - t0)
            if dt <= 0:
                break
            if dt > 2e-3:
                time.sleep(dt - 1e-3)
        tickets.append(srv.submit(probs[i]))
    lat, queue, ok, fin, sub = [], [], 0, [], []
    for t, k in zip(tickets, kinds):
        srv.wait(t, 3600.0)
        r, tm, _ = srv.result(t)
        lat.append(tm[2] - tm[0]); queue.append(tm[1] - tm[0]); fin.append(tm[2]); sub.append(tm[0])
        ok += r.status.name == "OPTIMAL"
    st = srv.stats()
    srv.close()
    lat = np.array(lat) * 1e3; queue = np.array(queue) * 1e3
    span = max(fin) - min(sub)
    sizes = [p.info()["n"] for p in probs[:nreq]]
    return {"offered_req_per_s": args.serve_rate, "requests": nreq, "solves_per_s": nreq / span,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())},
            "admission_wait_ms": {"p50": float(np.percentile(queue, 50)), "p99": float(np.percentile(queue, 99))},
            "optimal": f"{ok}/{nreq}", "grid_launches": st["launches"],
            "mix": "equal shares SOCP (SOC(20) blocks, m = 0.4 n), portfolio QP, max-cut SDP (one PSD block)",
            "sizes": f"target n log-uniform in [{args.serve_nmin}, {args.serve_nmax}], realised n in "
                     f"[{min(sizes)}, {max(sizes)}], mean {float(np.mean(sizes)):.0f}",
            "arena_gb": args.serve_arena_gb, "precision": args.precision}


def stable_arm(args, ctx):
    """The StableUzawaSolver factor against the default one on the same portfolio instances: one
    persistent launch per step, CUDA-event time, FP64."""
    from mumblebee_b200.ipm import Batch, IPMSettings
    probs, sizes = make_problems(args.extras_count, args.seed, 0, ctx)
    out = {"extra": "stable_factor", "workload": WORKLOAD, "instances": len(probs), "steps": args.steps,
           "warmup": args.warmup, "unit": "solves/s"}
    for name, st in (("default", IPMSettings()), ("stable", IPMSettings(stable=True))):
        batch = Batch(probs, st, ctx=ctx)
        for _ in range(args.warmup):
            batch.run()
        ms = [batch.run() for _ in range(args.steps)]
        res = batch.fetch(want_vectors=False)
        out[name] = {"solves_per_s": len(probs) / (statistics.mean(ms) / 1e3), "ms_per_step": statistics.mean(ms),
                     "optimal": sum(r.status.name == "OPTIMAL" for r in res),
                     "near_optimal": sum(r.status.name == "NEAR_OPTIMAL" for r in res),
                     "iters_mean": float(np.mean([r.niter for r in res])),
                     "factorizations_mean": float(np.mean([r.nfactor for r in res]))}
        del batch
    out["stable_over_default"] = out["stable"]["solves_per_s"] / out["default"]["solves_per_s"]
    print(json.dumps(out), flush=True)


def comp_arm(args, ctx):
    """extmul! with A and Aᵀ on a square block-sparse matrix of 4 x 4 blocks, up to 8 random
    target blocks per column block (N(0,1) entries), α = 1, β = 0: host-synchronous calls through
    the C ABI (b uploaded, c read back each call).  The kernel's own duration comes from an ncu
    launch list of the same command; the algorithmic bytes of one launch are printed for it."""
    from mumblebee_b200.comp import BlockSparseMatrix, extmul
    rng = np.random.default_rng(args.seed)
    nb, per = 4, 8
    n = args.comp_rows // nb * nb
    nblk = n // nb
    t = np.sort(rng.integers(0, nblk, size=(nblk, per)), axis=1)
    keep = np.ones_like(t, dtype=bool)
    keep[:, 1:] = np.diff(t, axis=1) > 0
    cnt = keep.sum(axis=1)
    tgt = t[keep]
    narc = int(tgt.size)
    xb = np.concatenate([[0], np.cumsum(cnt)])
    d = dict(nout=nblk, nvtx=nblk, narc=narc, ncol=n, nrow=n, nbnz=narc * nb * nb,
             xsrc=xb + 1, xcol=np.arange(nblk + 1, dtype=np.int64) * nb + 1,
             xrow=np.arange(nblk + 1, dtype=np.int64) * nb + 1,
             xblk=np.arange(narc + 1, dtype=np.int64) * nb * nb + 1, tgt=tgt + 1,
             val=rng.standard_normal(narc * nb * nb))
    t0 = time.time()
    A = BlockSparseMatrix(d, ctx=ctx)
    t_up = time.time() - t0
    b = rng.standard_normal(n)
    c = np.zeros(n)
    nnz = narc * nb * nb
    out = {"extra": "compensated_products", "kernel": "twomv_kernel", "rows": n, "cols": n, "stored_entries": nnz,
           "block": f"{nb}x{nb}, up to {per} target blocks per column block", "alpha": 1.0, "beta": 0.0,
           "upload_s": t_up, "calls": args.steps}
    for name, op, extra in (("A_b", A, 0), ("At_b", A.T, nnz)):
        for _ in range(args.warmup):
            extmul(c, op, b, 1.0, 0.0)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            extmul(c, op, b, 1.0, 0.0)
        sec = (time.perf_counter() - t0) / args.steps
        alg = 12 * nnz + extra + 8 * (n + 1) + 8 * n + 8 * n   # ptr, idx + val (+ block marks), b, c
        out[name] = {"call_ms": sec * 1e3, "algorithmic_bytes_per_launch": alg, "h2d_d2h_bytes_per_call": 16 * n}
    peaks = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    if os.path.exists(peaks):
        with open(peaks) as f:
            out["hbm_peak_gbs"] = {"value": json.load(f).get("hbm_gbs"), "source": "measured"}
    else:
        out["hbm_peak_gbs"] = {"value": 6650.0, "source": "fallback"}
    print(json.dumps(out), flush=True)


def coop_arm(args, ctx):
    """One SOCP instance (n = 2000, m = 800, 100 x SOC(20), density 0.0125, seed 0: one front of
    2000) solved once in the grid-cooperative mode (settings large = 1: CTA 0 runs the iteration,
    the other CTAs take the factor's tiles): the command behind the ipm_coop_kernel profile."""
    from mumblebee_b200 import generators as G
    from mumblebee_b200.ipm import Batch, IPMProblem, IPMSettings, _CONES
    pb = G.socp(2000, 800, 100, 0.0125, 0)
    prob = IPMProblem(pb["Q"], pb["B"], pb["f"], pb["g"], pb["mu"], [_CONES[k]() for k in pb["kinds"]], pb["sizes"],
                      ctx=ctx)
    batch = Batch([prob], IPMSettings(large=1), ctx=ctx)
    ms = batch.run()
    r = batch.fetch(want_vectors=False)[0]
    print(json.dumps({"extra": "coop_socp2000", "kernel": "ipm_coop_kernel", "ms": ms, "status": r.status.name,
                      "niter": r.niter, "nfactor": r.nfactor, "factor_flops": r.factor_flops}), flush=True)


def config4_arm(args, ctx):
    """The exponential/power-cone configuration: n = 20000 (3000 EXP, 1000 POW, 4000 free, 4000
    nonnegative columns), m = 5000, A at 0.1% density, seed 0, at the default 1e-8 tolerances,
    solved alone (grid-cooperative: its factorization exceeds the large-instance threshold).
    Wall time of init + solve; section clocks of the leader CTA; the last history rows."""
    from mumblebee_b200 import generators as G
    from mumblebee_b200.ipm import IPMProblem, IPMSettings, init, _CONES, PowerCone
    f = args.config4_scale
    pb = G.exppow(nexp=int(3000 * f), npow=int(1000 * f), nfree=int(4000 * f), npos=int(4000 * f), m=int(5000 * f),
                  density=0.001 / f)
    K = [PowerCone(a) if k == 5 else _CONES[k]() for k, a in zip(pb["kinds"], pb["params"])]
    t0 = time.time()
    prob = IPMProblem(pb["Q"], pb["B"], pb["f"], pb["g"], pb["mu"], K, pb["sizes"], ctx=ctx)
    sym = prob.symbolic()
    r_ = np.asarray(sym["nres"]) + np.asarray(sym["nsep"])
    t_sym = time.time() - t0
    clk = Clocks(0)
    t0 = time.time()
    s = init(prob, IPMSettings(precision=args.precision, fp32_tiles=args.fp32_tiles))
    r = s.solve()
    wall = time.time() - t0
    clocks = clk.stop()
    tm = s.timers()
    h = s.history()
    mhz = clocks.get("sm_mhz") or 1965.0
    fac_s = (tm["factor_update"] + tm["factor_diag"] + tm["factor_panel"]) / (mhz * 1e6)
    gap = (r.pobj - r.dobj) / max(1.0, min(abs(r.pobj), abs(r.dobj)))
    print(json.dumps({"extra": "config4_exppow", "precision": args.precision, "fp32_tiles": args.fp32_tiles,
                      "nfp32": r.nfp32, "nfallback": r.nfallback, "n": int(sum(pb["sizes"])), "m": int(pb["B"].shape[0]),
                      "fronts": int(sym["nfront"]), "largest_front": int(r_.max()), "symbolic_s": t_sym,
                      "status": r.status.name, "niter": r.niter, "pobj": r.pobj, "dobj": r.dobj, "rel_gap": gap,
                      "pres": r.pres, "dres": r.dres, "mu": r.mu, "nfactor": r.nfactor,
                      "nfactor_retry": r.nfactor_retry, "factor_flops": r.factor_flops, "wall_s": wall,
                      "factor_s": fac_s, "factor_tflops": r.nfactor * r.factor_flops / max(fac_s, 1e-9) / 1e12,
                      "sections_s": {k: v / (mhz * 1e6) for k, v in tm.items() if not k.startswith("n")},
                      "last_rows": [{k: h[i][k] for k in ("mu", "pres", "dres", "pobj", "dobj", "step", "rho")}
                                    for i in range(max(0, len(h) - 4), len(h))],
                      "clocks": clocks}), flush=True)


def main():
    args = parse()
    ws, rank, local, pg = dist_setup(args)
    if args.extras:
        from mumblebee_b200.ipm import Context
        ctx = Context.default(local)
        if args.extras in ("stable", "all"):
            stable_arm(args, ctx)
        if args.extras in ("comp", "all"):
            comp_arm(args, ctx)
        if args.extras in ("coop", "all"):
            coop_arm(args, ctx)
        if args.extras == "config4":
            config4_arm(args, ctx)
        return
    if args.impl == "reference":
        run_reference(args, ws, rank)
        if pg is not None:
            pg.destroy_process_group()
        return
    from mumblebee_b200.ipm import Context, IPMSettings, batch_solve
    ctx = Context.default(local)
    t0 = time.time()
    probs, sizes = make_problems(args.count, args.seed, rank, ctx)
    t_gen = time.time() - t0
    lower = lower_entries(probs)
    main_arm = timed_arm(probs, args.precision, args, pg, local, ws, ctx, lower)
    other = None
    if not args.no_compare:
        other = timed_arm(probs, "mixed" if args.precision == "fp64" else "fp64", args, pg, local, ws, ctx, lower)
    # roofline of the solver kernel: algorithmic factorization flops per launch / launch time, against
    # the FP64 GEMM peak (FP64 arm) and the TF32 tensor-core peak (FP32 / mixed arm)
    peaks = measure_peaks()

    def roof(arm):
        key = "fp64" if arm["precision"] == "fp64" else "tf32"
        achieved = arm["flops"] / (arm["ms"] / 1e3) / 1e12
        r = {"bound": "tensor", "achieved": achieved, "peak": peaks[key], "unit": "TFLOP/s",
             "frac": achieved / peaks[key], "traffic": None,
             "peak_source": f"measured live: torch {key} GEMM 8192^3 best of 5 on this GPU",
             "kernel": "ipm_batch_kernel", "precision": arm["precision"], "flops_per_launch": arm["flops"],
             "flops_fp32": arm["flops_fp32"], "flops_fp64": arm["flops_fp64"],
             "factorizations": arm["factorizations"], "alg_bytes": arm["alg_bytes"],
             "alg_bytes_source": "per factorization 8 B read (assembled B^T B) + 8 B (FP64) or 4 B (FP32) written "
                                 "per stored lower-triangle entry of L; per triangular-solve sweep one read of L",
             "hbm_achieved_gbs": arm["alg_bytes"] / (arm["ms"] / 1e3) / 1e9}
        if arm["precision"] == "fp64" and TRAFFIC_BYTES_PER_INSTANCE_FP64 is not None:
            r["traffic"] = TRAFFIC_BYTES_PER_INSTANCE_FP64 * args.count
            r["traffic_source"] = TRAFFIC_SOURCE
            r["traffic_over_alg"] = r["traffic"] / arm["alg_bytes"]
        return r

    roofline = roof(main_arm)
    roofline_other = roof(other) if other is not None else None
    # end to end through the C ABI: host problems in, host results out
    e2e = None
    if not args.no_e2e:
        # the main arm's launch configuration; a grid left to the library (0: two CTAs per SM in the
        # default build, one in the tensor-core build) keeps the call's chunked pipeline
        settings, grid = main_arm["settings"], main_arm["grid"]
        tuned = main_arm["autotune"]
        if tuned is None or tuned["choice"] in ("ffma_2_per_sm", "tcgen05_1_per_sm"):
            grid = 0
        batch_solve(probs, settings, grid=grid)          # warm-up
        barrier(pg, local)
        t = time.perf_counter()
        for _ in range(max(1, min(args.steps, 2))):
            batch_solve(probs, settings, grid=grid)
        dt = (time.perf_counter() - t) / max(1, min(args.steps, 2))
        dt = allreduce_max(pg, dt, local)
        st = main_arm["stats"]
        e2e = {"value": args.count * ws / dt, "unit": "solves/s", "h2d_bytes_per_step": st["input_bytes"],
               "d2h_bytes_per_step": st["output_bytes"],
               "note": "mb_batch_solve splits 1024+ problems into chunks planned and launched on their own "
                       "streams (planning overlaps device work); host symbolic analyses are cached by sparsity "
                       "structure and device blocks by the context, warm after the warm-up call"}
    serve = None
    if not args.no_serve:
        serve = serve_arm(args, ctx)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        k, ms, cores, sample = oracle_steps(args, 2, 1)
        cpu = {"value": k / (statistics.mean(ms) / 1e3), "unit": "solves/s", "cores": cores, "kind": "port",
               "sample": sample + "; 1 warm-up and 2 timed steps"}
    if rank == 0:
        st = main_arm["stats"]
        arms = {a["precision"]: {"solves_per_s": a["value"], "ms_per_step": a["ms_max"],
                                 "latency_ms": a["latency_ms"], "solve_ms": a["solve_ms"],
                                 "optimal": f"{a['optimal']}/{args.count}", "near_optimal": a["near_optimal"],
                                 "iters_mean": a["iters_mean"], "autotune": a["autotune"],
                                 "sections_mclk": a["sections_mclk"]}
                for a in (main_arm, other) if a is not None}
        if "mixed" in arms and "fp64" in arms:
            arms["mixed_over_fp64"] = arms["mixed"]["solves_per_s"] / arms["fp64"]["solves_per_s"]
        line = {"metric": METRIC, "value": main_arm["value"], "unit": "solves/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": main_arm["ms_max"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": main_config(args, ws),
                "footprint": {"input_gb": st["input_bytes"] / 1e9,
                              "workspace_gb": (st["work_bytes"] + st["factor_bytes"]) / 1e9},
                "run": {"optimal": f"{main_arm['optimal']}/{args.count}", "iters_mean": main_arm["iters_mean"],
                        "setup_s": {"generate": round(t_gen, 2), "prepare": round(main_arm["prepare_s"], 2)}},
                "latency_ms": main_arm["latency_ms"], "solve_ms": main_arm["solve_ms"],
                "precisions": arms, "serving": serve,
                "roofline": roofline, "roofline_other": roofline_other, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": args.steps,
                "clocks": main_arm["clocks"], "step_ms": main_arm["ms_steps"]}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
