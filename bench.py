#!/usr/bin/env python
"""bench.py — H-LU factor+solve/s at <= 1e-10 residual, mixed precision vs FP64.

Headline workload (the mixed-precision + iterative-refinement configuration): N = 65536 points
of U[0,1]^3 in Morton order, Laplace kernel 1/(4 pi (r + 1e-3)), diagonal shifted by 2 x the
largest off-diagonal row sum, standard admissibility eta = 1, leaf 512, adaptive rank <= 32 at
1e-8, 8 right-hand sides, refined in FP64 to a normwise backward error <= 1e-10.  The H-matrix is
built on the device from the points.  A "step" is one job: restore the matrix, factor, solve
and refine.  Two forms of the same job: the mixed form (Schur updates of the 512 leaves on the
tensor cores from BF16 shadows, FP32 accumulation; GETRF, TRSM, low-rank work and the refinement
residual in FP64) is the headline `value`; the plain FP64 form is timed beside it (`forms`).
Further legs: the FP64 HODLR batch (N = 8192, 64 jobs per merged launch), the serving loop.
Inputs are synthetic and seeded.  Multi-GPU: independent replicas, one per rank.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import importlib.util
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "H-LU factor+solve/s at 1e-10 residual, mixed vs FP64"
C3 = dict(n=65536, dim=3, kernel="laplace", p0=1e-3, leaf=512, admissibility=1, eta=1.0, kmax=32, rank_tol=1e-8,
          nrhs=8, tol=1e-10, seed=1234, gemm_tile=128)
C3_NAME = "laplace3d-n65536-leaf512-eta1-rank32tol1e-8-8rhs-bf16schur-fp64ir1e-10"
# the FP64 HODLR batch leg
WORKLOAD = dict(n=8192, dim=2, kernel="inv", p0=1e-3, leaf=256, rank=16, admissibility=0, seed=1234, tol=1e-10)
WORKLOAD_NAME = "hodlr-inv2d-n8192-leaf256-rank16-fp64-ir1e-10"
# DRAM bytes (read + write) of one job's factor work inside the batched HODLR factor launch, from
# one ncu capture of the batch-4 launch (dram__bytes.sum.per_second x gpu__time_duration.sum / 4);
# the jobs touch disjoint arenas, so the launch's traffic scales with the batch
FACTOR_DRAM_BYTES_PER_JOB = 117.5e6
# DRAM bytes (read + write) per algorithmic byte of the mixed factor launch of the headline job,
# from one ncu capture of the same launch at N = 16384 (28.2 GB read + 25.9 GB written against
# 72.9 GB of algorithmic bytes); the full-size launch's traffic is estimated by this ratio
C3_DRAM_PER_ALGORITHMIC_BYTE = (28.221709056e9 + 25.890199552e9) / 72.9413632e9


def load_pp():
    pkg = os.path.join(ROOT, "pastel-palettes_b200")
    spec = importlib.util.spec_from_file_location("pastel_palettes_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pastel_palettes_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
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
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = max(mx, float(f[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        except OSError:
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def program_bytes(pp, h, which=0, nrhs=1):
    """Compulsory operand bytes of one launch: targets read + written, inputs read once."""
    info = h.program_info(which, nrhs)
    tasks, _, _, _ = h.encode_program(which, nrhs, [0] * 5)
    total = 0
    for t in tasks:
        op, m, n, k, l = int(t["op"]), int(t["m"]), int(t["n"]), int(t["k"]), int(t["l"])
        if op == 1:
            e = 2 * m * n
        elif op in (2, 4, 5):
            e = 2 * m * n + m * m // 2
        elif op == 3:
            e = 2 * m * n + n * n // 2
        elif op == 6 and int(t["prec"]) == 2:  # BF16 shadows (2 bytes per element) into FP64 C; l: a
            # second operand pair summed in the same pass over C
            e = (2 if t["beta"] != 0 else 1) * m * n + (m * (k + l) + (k + l) * n) // 4
        elif op == 6:
            e = (2 if t["beta"] != 0 else 1) * m * n + m * k + k * n
        elif op == 9:
            e = 2 * (m * k + n * k) + (m + n) * l + n * k
        elif op == 10:
            e = (k + 2) * m * n
        elif op == 11:  # TRINV: leaf triangle read, an m x n column block of the inverse written
            e = m * m // 2 + m * n
        elif op == 12 and l > 0:  # TRMV part: its rows of the triangle and B read, l x n written
            o = int(t["o"])
            tri = sum((m - r) if int(t["ctrl"]) else (r + 1) for r in range(o, o + l))
            e = tri + m * n + l * n
        elif op == 12:  # TRMV: triangle read, B read and written
            e = m * m // 2 + 2 * m * n
        elif op in (13, 14):  # ORTH (in place) / COPY: m x n read and written
            e = 2 * m * n
        elif op == 15:  # SHADOW: m x k FP64 read, m x k BF16 written (split: m x k / 3 read)
            e = (m * k // 3 if int(t["o"]) else m * k) + m * k // 4
        else:
            e = 0
        total += 8 * e
    sel = (tasks["op"] == 6) & (tasks["prec"] == 2)
    kk = tasks["k"][sel].astype(np.int64) + tasks["l"][sel]
    info = dict(info, bf16_flops=float((2 * tasks["m"][sel].astype(np.int64) * tasks["n"][sel] * kk).sum()))
    return total, info


def whole_job_rate(dist, world, seconds, jobs_per_rank, device):
    """Whole-job throughput of `world` independent replicas: every rank processed
    `jobs_per_rank` jobs in `seconds` of its own device time, and the job ends with the slowest
    rank (max over ranks; the only collective of the bench).  Returns (jobs/s, max seconds)."""
    import torch
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return world * jobs_per_rank / t.item(), t.item()


def build_problem(pp, ctx, rank):
    w = WORKLOAD
    return pp.make_kernel_problem(ctx, w["n"], w["dim"], w["kernel"], w["p0"], w["leaf"], w["rank"],
                                  w["admissibility"], seed=w["seed"] + rank)


def fp64_peak_tflops(torch):
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


# ----------------------------------------------------------------------------- CPU arm
def reference_cpu_jobs(count, threads):
    """The reference's factor path on the host cores (oracle/hodlr.py, without this library): the
    workload's factorization program in the reference's instruction set (a committed fixture),
    executed by the oracle's restatement of the reference's block routines over its DAG with
    `threads` host threads, then the oracle's own substitution solve and FP64 refinement to the
    tolerance.  Each job restores the matrix first.  Returns (seconds per job, solves of the last
    job, the job object)."""
    import oracle.hodlr as oh
    job = oh.FixtureJob()
    A = job.dense()
    b = np.random.default_rng(7).uniform(-1.0, 1.0, (job.n, 1))
    times, hist = [], []
    for _ in range(count):
        t0 = time.perf_counter()
        _, hist = job.factor_solve(b, A, tol=WORKLOAD["tol"], threads=threads)
        times.append(time.perf_counter() - t0)
        if hist[-1] > WORKLOAD["tol"]:
            raise SystemExit(f"reference arm: refinement ended at {hist[-1]}")
    return times, len(hist), job


def config_keys(batch, precision, world):
    return {"workload": WORKLOAD_NAME, **WORKLOAD, "batch": batch, "precision": precision,
            "batch_note": "copies of one seeded matrix, distinct right-hand sides, one merged launch",
            "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas{world}"}


def run_reference_arm(args, rank, world):
    """The reference's CPU path on the headline job, on rank 0: each step one estimate of the job
    from the census sample (reference_c3_seconds); value = 1 / median."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    C3["n"] = args.n
    times, desc = [], ""
    for _ in range(args.warmup + args.steps):
        t, desc = reference_c3_seconds(threads)
        times.append(t)
    t = times[args.warmup:]
    value = 1.0 / float(np.median(t))
    line = {"metric": METRIC, "value": value, "unit": "factor+solve/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.median(t)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": c3_config_keys(world),
            "cpu_baseline": {"value": value, "unit": "factor+solve/s", "cores": threads, "kind": "port",
                             "sample": f"one estimate per step, value = 1 / median over {len(t)} steps: " + desc},
            "e2e": {"value": value, "unit": "factor+solve/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU arm
def make_batch(pp, ctx, batch, rank):
    """`batch` instances of the workload matrix (one seeded construction, copied into each
    instance's own host image and device arena); distinct right-hand sides per instance."""
    w = WORKLOAD
    h0, prob = build_problem(pp, ctx, rank)
    hs = [h0]
    for _ in range(1, batch):
        h = pp.Hierarchical.geometric(ctx, prob.points, w["leaf"], w["admissibility"], 1.0, w["rank"])
        h.host_arena()[:] = h0.host_arena()
        hs.append(h)
    return hs, [prob] * batch


def pipelined_e2e(pp, ctx, torch, hs, probs, b_host, bs, x_host, g_a, out_a, ref_a, batch_a, tune, iters, steps,
                  tol, s, barrier):
    """End-to-end throughput with the transfers overlapped: two device-resident input sets
    (the bench batch and a second copy) alternate; step k's matrices and right-hand sides go up
    on an upload stream while step k - 1 computes, its solutions come down on a download stream
    while step k + 1 computes.  Every step still moves its own inputs up from pinned host
    memory and its solutions down inside the timed region (first upload to last download).
    Returns (jobs of this rank, seconds, description)."""
    w = WORKLOAD
    hs_b = []
    for h in hs:
        q = pp.Hierarchical.geometric(ctx, probs[0].points, w["leaf"], w["admissibility"], 1.0, w["rank"])
        q.host_arena()[:] = h.host_arena()
        q.pin_host()
        q.upload(s)
        hs_b.append(q)
    s.synchronize()
    batch_b = pp.Batch(ctx, hs_b)
    if tune:
        batch_b.set_tuning(**tune)
    bs_b = [b.clone() for b in bs]
    x_host_b = [torch.empty_like(x).pin_memory() for x in x_host]
    ref_b = pp.BatchRefiner(batch_b, probs, stream=s)
    with torch.cuda.stream(s):
        batch_b.factor(s)
        ref_b.run(bs_b, iters)  # eager: allocates the plans before capture
        for q in hs_b:
            q.upload(s)
        g_b = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g_b, stream=s):
            batch_b.factor(s)
            out_b = ref_b.run(bs_b, iters)
    s.synchronize()
    sets = [(hs, bs, g_a, out_a, x_host, ref_a), (hs_b, bs_b, g_b, out_b, x_host_b, ref_b)]
    up_s, down_s = torch.cuda.Stream(), torch.cuda.Stream()
    ev = lambda: torch.cuda.Event(enable_timing=False)
    up, comp, down = [ev(), ev()], [ev(), ev()], [ev(), ev()]
    n_steps = 2 * max(2, steps)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(up_s)
    for k in range(n_steps):
        j = k % 2
        H, Bd, G, out, Xh, _ = sets[j]
        with torch.cuda.stream(up_s):
            if k >= 2:
                up_s.wait_event(down[j])  # the set's previous step has computed and come down
            for h in H:
                h.upload(up_s)
            for bd, bh in zip(Bd, b_host):
                bd.copy_(bh, non_blocking=True)
            up[j].record(up_s)
        with torch.cuda.stream(s):
            s.wait_event(up[j])
            G.replay()
            comp[j].record(s)
        with torch.cuda.stream(down_s):
            down_s.wait_event(comp[j])
            for xh, xd in zip(Xh, out[0]):
                xh.copy_(xd, non_blocking=True)
            down[j].record(down_s)
    up_s.wait_event(down[0])
    up_s.wait_event(down[1])
    e1.record(up_s)
    e1.synchronize()
    total = e0.elapsed_time(e1) / 1e3
    for H, Bd, G, out, Xh, ref in sets:
        if max(ref.errors(Bd, *out)) > tol:
            raise SystemExit("pipelined end-to-end step ended above the tolerance")
    mode = (f"{n_steps} steps over two alternating device input sets: uploads of step k overlap the "
            f"compute of step k - 1, downloads overlap step k + 1 (separate upload / download streams)")
    return len(hs) * n_steps, total, mode


def serving_leg(pp, ctx, n_requests, rates, seed=2024, smin=2048, smax=65536):
    """Poisson arrivals of factor+solve requests into the server (continuous admission), at each
    of the swept rates.  N log-uniform in [smin, smax] (multiple of 64), kernel uniform among
    Laplace 1/r, exp (length 0.1) and Matern-3/2 (length 0.2) on U[0,1]^3, weak admissibility,
    leaf 128, adaptive rank <= 32 at 1e-7, 1-16 right-hand sides, 0-4 follow-up sets reusing the
    resident factors, FP64 refinement to 1e-10.  Each request's H-matrix is built on the device at
    admission (inside its latency); the client computes the diagonal shift (device row sums)
    before submitting.  Latency = submission -> solutions on the host."""
    out = []
    for ri, rate in enumerate(rates):
        rng = np.random.default_rng(seed + 1000 * ri)
        kinds = [("laplace", 1e-3), ("exp", 0.1), ("matern32", 0.2)]
        reqs = []
        t_prep = time.perf_counter()
        for i in range(n_requests):
            n = int(round(np.exp(rng.uniform(np.log(smin), np.log(smax))) / 64)) * 64
            kern, p0 = kinds[int(rng.integers(0, 3))]
            nrhs = int(rng.integers(1, 17))
            sets = 1 + int(rng.integers(0, 5))
            h, prob = pp.make_kernel_problem(ctx, n, 3, kern, p0, 128, 32, seed=seed + 17 * i + ri, rank_tol=1e-7,
                                             construct="none")
            prob.points_dev = None
            reqs.append((h, prob, rng.uniform(-1, 1, (sets, n, nrhs))))
        t_prep = time.perf_counter() - t_prep
        gaps = rng.exponential(1.0 / rate, n_requests)
        srv = pp.Server(ctx, hbm_budget_bytes=96 << 30, max_inflight=4)
        # one untimed warm-up request (a server's first admission pays one-time host and driver setup)
        hw, pw = pp.make_kernel_problem(ctx, smin, 3, "laplace", 1e-3, 128, 32, seed=seed - 1, rank_tol=1e-7,
                                        construct="none")
        srv.submit(hw, pw, rng.uniform(-1, 1, (1, smin, 4)), tol=C3["tol"])
        srv.wait_all()
        ids, t0, t_next = [], time.perf_counter(), 0.0
        for (h, prob, rhs), g in zip(reqs, gaps):
            t_next += g
            delay = t_next - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            ids.append(srv.submit(h, prob, rhs, tol=C3["tol"]))
        srv.wait_all(timeout_ms=1800e3)
        st = [srv.poll(i) for i in ids]
        srv.close()
        if any(x["status"] != "done" for x in st):
            raise SystemExit(f"serving: a request failed: {[x['message'] for x in st if x['status'] != 'done'][:3]}")
        lat = np.array([x["t_done_ms"] - x["t_submit_ms"] for x in st])
        span_s = (max(x["t_done_ms"] for x in st) - min(x["t_submit_ms"] for x in st)) / 1e3
        vectors = sum(rhs.shape[0] * rhs.shape[2] for _, _, rhs in reqs)
        sizes = [p.n for _, p, _ in reqs]
        out.append({"arrival_rate_per_s": rate, "requests": n_requests, "p50_ms": float(np.percentile(lat, 50)),
                    "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                    "solves_per_s": vectors / span_s, "requests_per_s": n_requests / span_s,
                    "max_queued_ms": max(x["t_admit_ms"] - x["t_submit_ms"] for x in st),
                    "max_enqueue_ms": max(x["t_enqueued_ms"] - x["t_admit_ms"] for x in st),
                    "worst_backward_error": max(x["backward_error"] for x in st),
                    "refinement_solves": int(sum(x["iterations"] for x in st)), "n_median": float(np.median(sizes)),
                    "n_max": int(max(sizes)), "client_prep_s": t_prep})
    return {"rates": out, "solves_unit": "right-hand-side vectors solved to 1e-10 per second", "slots": 4,
            "workload": f"N log-uniform [{smin},{smax}] (multiple of 64), 3-D points, kernels laplace/exp/matern32, "
                        f"weak admissibility, leaf 128, adaptive rank <= 32 @ 1e-7, 1-16 RHS, 0-4 follow-up sets, "
                        f"Poisson arrivals; H-matrices built on the device at admission (inside the latency), the "
                        f"diagonal shift computed by the client before submission"}


def uneven_batch_leg(pp, ctx, n_inst, steps, warmup, seed=4096, smin=1024, smax=16384, restart=64):
    """Configuration-4 batch: n_inst H-matrices of uneven size in one merged persistent launch.
    N log-uniform in [smin, smax] (multiple of 64), points U[0,1]^2, kernel exp(-r / 0.1) + 1e-2 I,
    weak admissibility, leaf 128, adaptive rank at 1e-7 capped at 24, FP64 instructions (at leaf
    128 no Schur update qualifies for the BF16 form).  With these caps the H-LU is too coarse for
    plain refinement on the larger instances (rho(I - (LU)^-1 A) > 1: the blocks next to the
    diagonal need more rank than 24 at 1e-7), so the FP64 answer comes from restarted GMRES
    right-preconditioned by the batched H-LU solve (BatchGMRES: per step one merged solve launch,
    one batched matrix-free product, one Arnoldi launch; FP64 residual from the points at every
    restart) until every instance's backward error <= 1e-10.  Tile / grid autotuned; restore +
    factor + the GMRES cycles captured as one CUDA graph and replayed.  The matrices are built
    on the device before the clock."""
    import torch
    rng = np.random.default_rng(seed)
    hs, probs = [], []
    s = torch.cuda.Stream()
    t_build = time.perf_counter()
    with torch.cuda.stream(s):
        for i in range(n_inst):
            n = int(round(np.exp(rng.uniform(np.log(smin), np.log(smax))) / 64)) * 64
            h, prob = pp.make_kernel_problem(ctx, n, 2, "exp", 0.1, 128, 24, shift=1e-2, seed=seed + 31 * i,
                                             rank_tol=1e-7, construct="device", stream=s)
            h.keep_original(s)
            hs.append(h)
            probs.append(prob)
    s.synchronize()
    t_build = time.perf_counter() - t_build
    batch = pp.Batch(ctx, hs)
    tune = batch.autotune(s)
    bs = [torch.from_numpy(pp.rhs(p.n, 1, seed=3 + i)).cuda() for i, p in enumerate(probs)]
    # plain refinement first, for the record: where it stalls
    ir = pp.BatchRefiner(batch, probs, stream=s)
    with torch.cuda.stream(s):
        batch.restore(s)
        batch.factor(s)
        _, ir_hist = ir.solve(bs, tol=WORKLOAD["tol"], max_iter=10)
    gm = pp.BatchGMRES(batch, probs, m=restart, stream=s, lowp=True)
    t_warm = time.perf_counter()
    with torch.cuda.stream(s):
        for _ in range(max(1, warmup)):
            batch.restore(s)
            batch.factor(s)
            _, hist = gm.solve(bs, tol=WORKLOAD["tol"], max_cycles=40)
    batch.sync(s)
    t_warm = (time.perf_counter() - t_warm) / max(1, warmup)
    cycles = len(hist)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            batch.restore(s)
            batch.factor(s)
            out = gm.run(bs, cycles)
    total, worst = 0.0, 0.0
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(s):
            e0.record(s)
            g.replay()
            e1.record(s)
        e1.synchronize()
        total += e0.elapsed_time(e1) / 1e3
        worst = max(worst, max(gm.errors(bs, *out)))
    batch.sync(s)
    # factor alone, for the split of the step
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(s):
        batch.restore(s)
        f0.record(s)
        batch.factor(s)
        f1.record(s)
    f1.synchronize()
    converged = worst <= WORKLOAD["tol"]
    sizes = [p.n for p in probs]
    flops = batch.program_info(0)["flops"]
    del g
    return {"converged_to_tol": converged, "instances": n_inst, "n_min": min(sizes), "n_max": max(sizes),
            "n_total": int(sum(sizes)), "factor_solve_per_s": n_inst * steps / total,
            "ms_per_step": 1e3 * total / steps, "factor_ms": f0.elapsed_time(f1),
            "gmres_cycles": cycles, "gmres_restart": restart, "krylov_steps": cycles * restart,
            "gmres_history": hist, "worst_backward_error": worst,
            "plain_refinement_backward_error_after_10": ir_hist[-1],
            "factor_gflop_per_step": flops / 1e9, "factor_gflops": flops / (f0.elapsed_time(f1) / 1e3) / 1e9,
            "eager_step_s": t_warm, "autotune": tune, "construction_s": t_build,
            "workload": "N log-uniform [1024,16384], exp(-r/0.1)+1e-2 I on U[0,1]^2, weak admissibility, leaf 128, "
                        "adaptive rank @ 1e-7 capped at 24, built on the device before the clock, FP64 "
                        "instructions (no leaf qualifies for the BF16 form); FP64 answer by restarted GMRES "
                        f"(restart {restart}) right-preconditioned by the merged H-LU solve, products inside a "
                        "cycle with FP32-evaluated kernel entries, FP64 residual from the points at every restart "
                        "(the convergence test); restore + factor + GMRES captured as one CUDA graph"}


# ----------------------------------------------------------------------------- headline job
def c3_config_keys(world):
    return {"workload": C3_NAME, **C3, "batch": 1,
            "precision": "mixed: bf16 schur updates of the 512 leaves (fp32 accumulation); fp64 getrf, trsm, "
                         "low-rank work and refinement residual",
            "comparison": "plain fp64 form of the same job (forms.fp64)",
            "construction": "on the device from the points (dense blocks assembled, low-rank blocks by a "
                            "randomized range finder), before the clock for value, inside it for e2e",
            "l2": "not flushed: the 29 GB matrix and its 29 GB original are far larger than L2",
            "parallelism": f"replicas{world}"}


class C3Job:
    """One job of the headline workload on this rank's GPU (seed offset by rank): the H-matrix built
    on the device from its points, its original kept for restores, 8 right-hand sides."""

    def __init__(self, pp, ctx, torch, s, rank):
        self.pp, self.ctx, self.torch, self.s = pp, ctx, torch, s
        c = C3
        t0 = time.perf_counter()
        with torch.cuda.stream(s):
            self.h, self.prob = pp.make_kernel_problem(ctx, c["n"], c["dim"], c["kernel"], c["p0"], c["leaf"],
                                                       c["kmax"], c["admissibility"], c["eta"], seed=c["seed"] + rank,
                                                       rank_tol=c["rank_tol"], construct="device", stream=s)
            self.h.sync(s)
            self.h.keep_original(s)
        s.synchronize()
        self.setup_s = time.perf_counter() - t0
        self.h.set_gemm_tile(c["gemm_tile"])
        self.b = torch.from_numpy(pp.rhs(c["n"], c["nrhs"], seed=7 + rank)).cuda()
        self.rank = rank

    def run_form(self, prec, steps, warmup, barrier):
        """restore + factor + refinement to the tolerance, device-timed per step (CUDA events on
        the job's stream); the factor launch is timed inside the same steps."""
        pp, torch, h, s = self.pp, self.torch, self.h, self.s
        h.set_precision(prec)
        t0 = time.perf_counter()
        info = h.program_info(0)
        build_s = time.perf_counter() - t0
        dag_ms, dag_dev = h.dag_info(0)
        fbytes, finfo = program_bytes(pp, h, 0)
        ref = pp.Refiner(h, self.ctx, self.prob, stream=s)
        tol = C3["tol"]
        with torch.cuda.stream(s):
            for _ in range(warmup):
                h.restore(s)
                h.factor(s)
                ref.solve(self.b, tol=tol)
        h.sync(s)
        barrier()
        l0 = ref.launches
        tot, fac, rfn, worst, iters = 0.0, [], [], 0.0, 0
        for _ in range(steps):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            with torch.cuda.stream(s):
                ev[0].record(s)
                h.restore(s)
                ev[1].record(s)
                h.factor(s)
                ev[2].record(s)
                _, hist = ref.solve(self.b, tol=tol)
                ev[3].record(s)
            ev[3].synchronize()
            tot += ev[0].elapsed_time(ev[3]) / 1e3
            fac.append(ev[1].elapsed_time(ev[2]))
            rfn.append(ev[2].elapsed_time(ev[3]))
            worst = max(worst, hist[-1])
            iters = len(hist)
        h.sync(s)
        barrier()
        if worst > tol:
            raise SystemExit(f"a timed step ended above {tol}: {worst}")
        return {"total_s": tot, "ms_per_step": 1e3 * tot / steps, "steps": steps, "warmup": warmup,
                "factor_ms": float(np.median(fac)), "refine_ms": float(np.median(rfn)), "refinement_solves": iters,
                "worst_backward_error": worst, "factor_tasks": info["n_tasks"], "factor_flops": info["flops"],
                "factor_bytes": fbytes, "bf16_flops": finfo["bf16_flops"], "program_build_s": build_s,
                "dag_build_ms": dag_ms, "dag_built_on_device": dag_dev,
                "gpu_launches_per_step": 2 + (ref.launches - l0) / max(1, steps)}

    def e2e(self, prec, steps, barrier):
        """End to end from host buffers: points and right-hand sides up from pinned host memory,
        the off-diagonal row sums (diagonal shift), the H-matrix built on the device, factor,
        refinement, solutions down; one warm-up step, then `steps` timed."""
        pp, torch, h, s, prob = self.pp, self.torch, self.h, self.s, self.prob
        h.set_precision(prec)
        pts_host = torch.from_numpy(np.ascontiguousarray(prob.points)).pin_memory()
        b_host = self.b.cpu().pin_memory()
        x_host = torch.empty_like(b_host).pin_memory()
        pts_dev = torch.empty(pts_host.shape, dtype=torch.float64, device="cuda")
        b_dev = torch.empty(b_host.shape, dtype=torch.float64, device="cuda")
        ref = pp.Refiner(h, self.ctx, prob, stream=s)
        tot = 0.0
        barrier()
        for i in range(steps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s):
                e0.record(s)
                pts_dev.copy_(pts_host, non_blocking=True)
                b_dev.copy_(b_host, non_blocking=True)
                off = pp.offdiag_rowsum_max_dev(self.ctx, pts_dev, prob.kernel, prob.p0, s)
                if abs(2.0 * off - prob.shift) > 1e-9 * prob.shift:
                    raise SystemExit("e2e: the diagonal shift differs from the job's")
                h.construct(prob, pts_dev, s)
                h.factor(s)
                x, hist = ref.solve(b_dev, tol=C3["tol"])
                x_host.copy_(x, non_blocking=True)
                e1.record(s)
            e1.synchronize()
            if hist[-1] > C3["tol"]:
                raise SystemExit("e2e step ended above the tolerance")
            if i > 0:
                tot += e0.elapsed_time(e1) / 1e3
        h.sync(s)
        barrier()
        # leave the matrix as the other forms expect it: the original is still kept on the device
        n, d, r = prob.n, prob.dim, self.b.shape[1]
        return {"total_s": tot, "steps": steps, "h2d": 8 * n * (d + r), "d2h": 8 * n * r,
                "mode": "one job at a time through the C ABI: points and right-hand sides up from pinned host "
                        "memory, row sums for the diagonal shift, H-matrix built on the device (dense blocks "
                        "assembled, low-rank blocks compressed), mixed factor, FP64 refinement, solutions down"}

    def roofline(self, mixed, fp64):
        hbm_peak, peak_kind = peaks()
        fac_s = mixed["factor_ms"] / 1e3
        achieved = mixed["factor_bytes"] / fac_s / 1e9
        out = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
               "traffic": C3_DRAM_PER_ALGORITHMIC_BYTE * mixed["factor_bytes"],
               "traffic_source": "ncu DRAM bytes of the same launch at N = 16384 (0.74 per algorithmic byte), scaled "
                                 "by the algorithmic bytes of this launch",
               "kernel": "vm_kernel (mixed factor launch, one job)", "launch_ms": 1e3 * fac_s,
               "algorithmic_bytes": mixed["factor_bytes"],
               "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"}
        bf16_peak = bf16_peak_tflops()
        tc = mixed["bf16_flops"] / fac_s / 1e12
        out["tensor"] = {"achieved_tflops": tc, "peak_tflops": bf16_peak, "frac": tc / bf16_peak,
                         "flops": mixed["bf16_flops"], "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained "
                                                                      "(the launch runs for seconds)"}
        if fp64:
            fp64_peak = fp64_peak_tflops(self.torch)
            f = fp64["factor_flops"] / (fp64["factor_ms"] / 1e3) / 1e12
            out["fp64_form"] = {"achieved_tflops": f, "peak_tflops": fp64_peak, "frac": f / fp64_peak,
                                "launch_ms": fp64["factor_ms"],
                                "peak_source": "measured in this run: torch float64 matmul 8192^3"}
        return out

    def release(self):
        """Frees the job's device memory (the matrix, its original and the plans)."""
        self.h = self.prob = self.b = None
        import gc
        gc.collect()
        self.torch.cuda.empty_cache()


def bf16_peak_tflops():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("bf16_tflops_sustained", d.get("bf16_tflops", 1400.0))
    return 1400.0


def reference_c3_seconds(threads):
    """The reference's CPU path on the headline job, estimated from a bounded sample: every
    instruction class of the job's plain FP64 factorization and solve programs (the census
    fixture) timed on the oracle's restated reference routines and weighted by its count, plus one
    FP64 matrix-free residual (timed on a 1024-row slab of the kernel matrix times the 8 right-hand
    sides, scaled to N rows); one refinement solve, as the FP64 form needs.  Host threads assumed
    to scale ideally.  Returns (seconds per job, description)."""
    import oracle.census as oc
    from oracle.hodlr import distances, kernel_eval
    tf, d0 = oc.program_seconds(0, threads)
    ts, d1 = oc.program_seconds(1, threads)
    n, nrhs = C3["n"], C3["nrhs"]
    rng = np.random.default_rng(C3["seed"])
    pts = rng.uniform(0.0, 1.0, (n, C3["dim"]))
    x = rng.standard_normal((n, nrhs))
    slab = 1024
    t0 = time.perf_counter()
    K = kernel_eval(1, distances(pts[:slab], pts), C3["p0"])
    _ = K @ x
    tr = (time.perf_counter() - t0) * (n / slab) / threads
    total = tf + ts + tr
    desc = (f"estimate from a bounded sample ({threads} threads assumed to scale ideally): the job's FP64 "
            f"factor program ({d0['instructions']} instructions in {d0['classes']} classes, "
            f"{d0['flops'] / 1e12:.1f} TFLOP) and 8-RHS solve program ({d1['instructions']} instructions) from "
            f"tests/golden/c3_census.npz, every class timed once on the oracle's restated reference routines "
            f"and weighted by its count ({tf:.0f} s + {ts:.1f} s), plus one residual from a timed 1024-row slab "
            f"of the kernel matrix ({tr:.1f} s)")
    return total, desc


def c2_batch_leg(args, pp, ctx, torch, dist, rank, world, barrier, s):
    """The FP64 HODLR batch: 64 jobs of the N = 8192 configuration (copies of one seeded matrix,
    distinct right-hand sides) per merged persistent launch; restore + factor + refinement solves
    captured as one CUDA graph and replayed; L2 flushed between steps.  Returns its JSON object."""
    tol = WORKLOAD["tol"]
    B = args.batch
    hs, probs = make_batch(pp, ctx, B, rank)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        for h in hs:
            h.pin_host()
            h.upload(s)
            h.keep_original(s)
    s.synchronize()
    n = probs[0].n
    b_host = [torch.from_numpy(pp.rhs(n, 1, seed=7 + i)).pin_memory() for i in range(B)]
    bs = [x.cuda() for x in b_host]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2

    def run_form(prec, clk=None):
        """Device-timed steps of one precision form: batched restore + factor + refinement
        solves captured as one CUDA graph.  Returns (batch, refiner, graph, outputs, stats)."""
        for h in hs:
            h.set_precision(prec)
            if args.gemm_tile and not args.autotune:
                h.set_gemm_tile(args.gemm_tile)
        batch = pp.Batch(ctx, hs)
        tune = batch.autotune(s) if args.autotune else None
        ref = pp.BatchRefiner(batch, probs, stream=s)
        # warm-up (eager): allocates every plan, fixes the number of refinement solves
        with torch.cuda.stream(s):
            for _ in range(args.warmup):
                batch.restore(s)
                batch.factor(s)
                xs, hist = ref.solve(bs, tol=tol)
        batch.sync(s)
        if hist[-1] > tol:
            raise SystemExit(f"refinement did not reach {tol}: {hist}")
        iters = len(hist)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                batch.restore(s)
                batch.factor(s)
                out = ref.run(bs, iters)
        total, worst = 0.0, 0.0
        barrier()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s):  # replay on the stream the events are recorded on
                e0.record(s)
                g.replay()
                e1.record(s)
            e1.synchronize()
            total += e0.elapsed_time(e1) / 1e3
            worst = max(worst, max(ref.errors(bs, *out)))
        barrier()
        batch.sync(s)
        if worst > tol:
            raise SystemExit(f"a timed step ended above {tol}: {worst}")
        value, total_max = whole_job_rate(dist, world, total, B * args.steps, "cuda")
        stats = {"value": value, "ms_per_step": 1e3 * total_max / args.steps,
                 "refinement_solves": iters, "worst_backward_error": worst, "total_s": total_max,
                 "autotune": tune}
        return batch, ref, g, out, stats

    forms = {"fp64": pp.FP64, "tf32": pp.TF32}
    other = "fp64" if args.precision == "tf32" else "tf32"
    # the comparison form first, then the headline form (whose plans the rest reuses)
    cmp_stats = None
    if args.compare:
        bt, _, gc, _, cmp_stats = run_form(forms[other])
        del gc, bt
    batch, ref, g, out, main_stats = run_form(forms[args.precision])
    iters = main_stats["refinement_solves"]
    total_max = main_stats["total_s"]
    value = main_stats["value"]
    # per step: the factor (init + VM), per refinement iteration one batched solve (init + VM)
    # and the batched update / residual / reduction launches
    launches_per_step = 2 + iters * (2 + pp.residual_batch_launches(
        [(p.kernel, p.dim, b.shape[1], True) for p, b in zip(probs, bs)]))

    # --- end to end through the C ABI: matrices and right-hand sides up from pinned host
    #     memory, batched factor + refinement, solutions down
    g2 = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g2, stream=s):
            batch.factor(s)
            out2 = ref.run(bs, iters)
    x_host = [torch.empty_like(x).pin_memory() for x in b_host]
    e2e_steps = max(3, args.steps // 2)
    e2e_total = 0.0
    barrier()
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(s):
            e0.record(s)
            for h in hs:
                h.upload(s)
            for bd, bh in zip(bs, b_host):
                bd.copy_(bh, non_blocking=True)
            g2.replay()
            for xh, xd in zip(x_host, out2[0]):
                xh.copy_(xd, non_blocking=True)
        e1.record(s)
        e1.synchronize()
        e2e_total += e0.elapsed_time(e1) / 1e3
    if max(ref.errors(bs, *out2)) > tol:
        raise SystemExit("end-to-end step ended above the tolerance")
    e2e_serial, _ = whole_job_rate(dist, world, e2e_total, B * e2e_steps, "cuda")
    e2e_jobs, e2e_seconds, e2e_mode = pipelined_e2e(pp, ctx, torch, hs, probs, b_host, bs, x_host, g2, out2, ref,
                                                    batch, main_stats["autotune"], iters, e2e_steps, tol, s, barrier)
    e2e_value, _ = whole_job_rate(dist, world, e2e_seconds, e2e_jobs, "cuda")

    # --- the dominant kernel (the batched factor launch), timed alone
    fac_ms = []
    with torch.cuda.stream(s):
        for _ in range(args.steps):
            batch.restore(s)
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            batch.factor(s)
            e1.record(s)
            e1.synchronize()
            fac_ms.append(e0.elapsed_time(e1))
    batch.sync(s)
    # one job alone (latency of a single factor+solve, eager with adaptive refinement)
    single = pp.Batch(ctx, [hs[0]])
    ref1 = pp.BatchRefiner(single, probs[:1], stream=s)
    lat = []
    with torch.cuda.stream(s):
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            single.restore(s)
            single.factor(s)
            ref1.solve(bs[:1], tol=tol)
            e1.record(s)
            e1.synchronize()
            lat.append(e0.elapsed_time(e1))
    fbytes, finfo = program_bytes(pp, hs[0], 0)
    hbm_peak, peak_kind = peaks()
    fac_s = float(np.median(fac_ms)) / 1e3
    fp64_peak = fp64_peak_tflops(torch)
    achieved_gbs = B * fbytes / fac_s / 1e9
    roofline = {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved_gbs / hbm_peak, "traffic": B * FACTOR_DRAM_BYTES_PER_JOB,
                "traffic_source": "ncu capture of the batch-4 factor launch, scaled by jobs per launch",
                "kernel": f"vm_kernel (batched factor launch, {B} jobs)", "launch_ms": 1e3 * fac_s,
                "algorithmic_bytes": B * fbytes, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "fp64": {"achieved_tflops": B * finfo["flops"] / fac_s / 1e12, "peak_tflops": fp64_peak,
                         "frac": B * finfo["flops"] / fac_s / 1e12 / fp64_peak,
                         "peak_source": "measured in this run: torch float64 matmul 8192^3"}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        times, its, job = reference_cpu_jobs(6, threads)
        cpu = {"value": 1.0 / float(np.median(times[1:])), "unit": "factor+solve/s", "cores": threads, "kind": "port",
               "sample": f"5 jobs of the workload after 1 warm-up, value = 1 / median: the reference-ISA factor "
                         f"program on the oracle's restated reference routines over its DAG ({threads} threads), "
                         f"the oracle's substitution solve, FP64 refinement ({its} solves)"}
    del g, g2
    return {"metric": "H-LU factor+solve/s at 1e-10 residual (FP64 HODLR N=8192, batch of 64)", "value": value,
            "unit": "factor+solve/s", "ms_per_step": 1e3 * total_max / args.steps, "steps": args.steps,
            "forms": {args.precision: {k: v for k, v in main_stats.items() if k != "total_s"},
                      **({other: {k: v for k, v in cmp_stats.items() if k != "total_s"}} if cmp_stats else {})},
            "config": config_keys(B, args.precision, world),
            "details": {"graph": "restore+factor+solves captured", "factor_tasks_per_job": finfo["n_tasks"],
                        "factor_flops_per_job": finfo["flops"], "refinement_solves": iters,
                        "single_job_step_ms": float(np.median(lat))},
            "e2e": {"value": e2e_value, "unit": "factor+solve/s", "h2d_bytes_per_step": B * (hs[0].arena_bytes() + 8 * n),
                    "d2h_bytes_per_step": B * 8 * n, "mode": e2e_mode, "serial_value": e2e_serial,
                    "serial_mode": "one step at a time: upload, factor + refinement, download, then the next"},
            "roofline": roofline, "cpu_baseline": cpu,
            "plain_fp64_single_instance": {
                "value": 1e3 / float(np.median(lat)), "unit": "factor+solve/s",
                "note": "one job per persistent launch, FP64, refinement to the same tolerance (the reference's "
                        "execution model: one DAG per launch)"},
            "gpu_launches_per_step": launches_per_step}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fp64-steps", type=int, default=2, help="timed steps of the plain FP64 comparison form "
                                                              "(after one warm-up step; 0: skip)")
    ap.add_argument("--n", type=int, default=C3["n"], help="points of the headline workload (smaller: quick runs)")
    ap.add_argument("--batch", type=int, default=64, help="jobs per merged launch of the HODLR batch leg (0: skip)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "tf32"], help="HODLR batch leg: headline form")
    ap.add_argument("--compare", type=int, default=0, help="HODLR batch leg: also time the other precision form")
    ap.add_argument("--autotune", type=int, default=1, help="HODLR batch leg: pick tile and grid by timing")
    ap.add_argument("--gemm-tile", type=int, default=0, help="HODLR batch leg: product tile edge when not tuning")
    ap.add_argument("--serve-requests", type=int, default=200, help="requests per rate of the serving leg (0: skip)")
    ap.add_argument("--serve-rates", default="2,4,8", help="Poisson arrival rates of the serving leg (1/s)")
    ap.add_argument("--uneven", type=int, default=512, help="instances of the uneven batch leg (0: skip)")
    args = ap.parse_args()
    C3["n"] = args.n
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":  # the oracle alone: this library is not loaded
        run_reference_arm(args, rank, world)
        return
    pp = load_pp()

    import torch
    import torch.distributed as dist
    from datetime import timedelta
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    ctx = pp.Context(device=local)
    ctx.set_device_dag(True)  # dependency DAGs of the programs built on the GPU (same DAG as the host's)
    s = torch.cuda.Stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    t_start = time.perf_counter()
    job = C3Job(pp, ctx, torch, s, rank)
    with Clocks(local) as clk:
        mixed = job.run_form(pp.BF16, args.steps, args.warmup, barrier)
    value, total_max = whole_job_rate(dist, world, mixed["total_s"], args.steps, "cuda")
    fp64 = None
    if args.fp64_steps > 0:
        fp64 = job.run_form(pp.FP64, args.fp64_steps, 1, barrier)
        fp64["value"], fp64["total_s"] = whole_job_rate(dist, world, fp64["total_s"], args.fp64_steps, "cuda")
    e2e = job.e2e(pp.BF16, max(2, args.steps // 2), barrier)
    e2e_value, _ = whole_job_rate(dist, world, e2e["total_s"], e2e["steps"], "cuda")
    roofline = job.roofline(mixed, fp64)
    c3_config = c3_config_keys(world)
    job.release()
    print(f"bench: headline job {time.perf_counter() - t_start:.0f} s", file=sys.stderr, flush=True)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t_est, sample = reference_c3_seconds(os.cpu_count() or 1)
        cpu = {"value": 1.0 / t_est, "unit": "factor+solve/s", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": sample}
    legs = {}
    if world > 1:  # the legs are single-GPU measurements; replicas run the headline job only
        args.batch = args.uneven = args.serve_requests = 0
    t_leg = time.perf_counter()
    if args.batch > 0:
        legs["hodlr_batch"] = c2_batch_leg(args, pp, ctx, torch, dist, rank, world, barrier, s)
        print(f"bench: hodlr batch leg {time.perf_counter() - t_leg:.0f} s", file=sys.stderr, flush=True)
    t_leg = time.perf_counter()
    if args.uneven > 0:
        legs["uneven_batch"] = uneven_batch_leg(pp, ctx, args.uneven, 3, 1)
        print(f"bench: uneven batch leg {time.perf_counter() - t_leg:.0f} s", file=sys.stderr, flush=True)
    t_leg = time.perf_counter()
    # admission builds programs while other requests' persistent launches hold every SM: a
    # DAG build on the device would queue behind them, so the server builds on the host
    ctx.set_device_dag(False)
    if args.serve_requests > 0:
        legs["serving"] = serving_leg(pp, ctx, args.serve_requests, [float(x) for x in args.serve_rates.split(",")],
                                      seed=2024 + rank)
        print(f"bench: serving leg {time.perf_counter() - t_leg:.0f} s", file=sys.stderr, flush=True)

    if rank == 0:
        forms = {"bf16": {k: v for k, v in mixed.items() if k != "total_s"}}
        forms["bf16"]["value"] = value
        if fp64:
            forms["fp64"] = {k: v for k, v in fp64.items() if k != "total_s"}
        line = {"metric": METRIC, "value": value, "unit": "factor+solve/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * total_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "bf16 schur + f64", "data": "synthetic",
                "config": c3_config, "forms": forms,
                "mixed_vs_fp64": (value / fp64["value"]) if fp64 else None,
                "e2e": {"value": e2e_value, "unit": "factor+solve/s", "h2d_bytes_per_step": e2e["h2d"],
                        "d2h_bytes_per_step": e2e["d2h"], "mode": e2e["mode"]},
                "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(), "legs": legs,
                "gpu_launches": mixed["gpu_launches_per_step"] * args.steps}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
