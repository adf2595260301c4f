#!/usr/bin/env python
"""trace_tool.py — per-instruction trace of the VM and its critical-path analysis.

Counterpart of the reference's clock tracing (every instruction stamps clock64 at start and
end, src/kernel.cu:1389-1390, rendered per worker by analyzeClocks, rts/scheduler.cpp:494-544).
Here the VM stamps the globaltimer (ns) at a task's start and end plus its SM and CTA
(`pp_hmatrix_trace` / `pp_batch_trace`); this tool runs a HODLR workload with tracing on and
reports, per program (factor, solve):

  * makespan, CTAs used, busy time and the average parallelism (busy / makespan);
  * busy time per instruction shape (op, m, n, k);
  * the critical path recomputed from the measured durations over the program's DAG edges,
    its composition by instruction shape, and the waits between consecutive path tasks;
  * the ready-to-start latency (a task's start minus its last predecessor's end).

  python pastel-palettes_b200/trace_tool.py [--n 8192] [--leaf 256] [--rank 16] [--batch 16]
                                            [--gemm-tile 64|128] [--out trace.npz]
  python pastel-palettes_b200/trace_tool.py --workload laplace3d [--n 65536] [--form bf16|fp64]
      the mixed-precision configuration instead (3-D Laplace, leaf 512, eta 1, adaptive rank
      <= 32 at 1e-8, built on the device): its factor and its 8-RHS solve
  python pastel-palettes_b200/trace_tool.py --workload gmres [--instances 512] [--restart 32]
      device times of the parts of one GMRES step over the uneven batch
  python pastel-palettes_b200/trace_tool.py --workload dag [--n 65536]
      the mixed configuration's factor program DAG built on the host and on the device
"""
import argparse
import collections
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _load():
    if "pastel_palettes_b200" in sys.modules:
        return sys.modules["pastel_palettes_b200"]
    spec = importlib.util.spec_from_file_location("pastel_palettes_b200", os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pastel_palettes_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def critical_path(dur, start, preds):
    """Longest path by measured durations (tasks visited in start order, a topological order
    of an executed DAG); returns (length, path as task ids from sink to source)."""
    fin, arg = {}, {}
    for i in np.argsort(start, kind="stable"):
        i = int(i)
        best, bp = 0, -1
        for p in preds[i]:
            if fin.get(p, 0) > best:
                best, bp = fin[p], p
        fin[i] = int(dur[i]) + best
        arg[i] = bp
    i = max(fin, key=fin.get)
    path = []
    while i >= 0:
        path.append(i)
        i = arg[i]
    return max(fin.values()), path


def analyse(name, tasks, trace, ef, et, out=print):
    ops = _load().OP_NAMES
    st, en = trace[:, 0].astype(np.int64), trace[:, 1].astype(np.int64)
    cta = trace[:, 2].astype(np.int64) >> 32
    dur = en - st
    mk = en.max() - st.min()
    out(f"== {name}: tasks {len(tasks)} makespan {mk / 1e3:.1f} us, CTAs used {len(np.unique(cta))}")
    out(f"   busy {dur.sum() / 1e3:.1f} us -> average parallelism {dur.sum() / mk:.1f}")
    agg = collections.defaultdict(list)
    for i in range(len(tasks)):
        agg[(ops[tasks["op"][i]], int(tasks["m"][i]), int(tasks["n"][i]), int(tasks["k"][i]))].append(dur[i])
    out(f"   {'op, m, n, k':34s} {'count':>6s} {'mean us':>8s} {'total us':>9s} {'share':>6s}")
    for k, v in sorted(agg.items(), key=lambda x: -sum(x[1]))[:16]:
        out(f"   {str(k):34s} {len(v):6d} {np.mean(v) / 1e3:8.2f} {sum(v) / 1e3:9.1f} {100 * sum(v) / dur.sum():5.1f}%")
    preds = collections.defaultdict(list)
    for a, b in zip(ef, et):
        preds[int(b)].append(int(a))
    cp, path = critical_path(dur, st, preds)
    gaps = sum(max(0, st[path[j]] - en[path[j + 1]]) for j in range(len(path) - 1))
    out(f"   critical path {cp / 1e3:.1f} us over {len(path)} tasks ({cp / mk:.2f} of the makespan), "
        f"waits between path tasks {gaps / 1e3:.0f} us")
    comp = collections.defaultdict(lambda: [0, 0])
    for i in path:
        k = (ops[tasks["op"][i]], int(tasks["m"][i]), int(tasks["n"][i]), int(tasks["k"][i]))
        comp[k][0] += 1
        comp[k][1] += dur[i]
    for k, v in sorted(comp.items(), key=lambda x: -x[1][1])[:10]:
        out(f"     on path: {str(k):34s} {v[0]:4d} tasks {v[1] / 1e3:9.1f} us")
    lat = [st[i] - max(en[p] for p in preds[i]) for i in range(len(tasks)) if preds[i]]
    if lat:
        out(f"   ready->start latency: median {np.median(lat) / 1e3:.2f} us, p90 {np.percentile(lat, 90) / 1e3:.2f} us")


def trace_laplace3d(pp, ctx, torch, args):
    """Factor and 8-RHS solve of the mixed-precision configuration, traced."""
    n = args.n if args.n != 8192 else 65536
    h, prob = pp.make_kernel_problem(ctx, n, 3, "laplace", 1e-3, 512, 32, admissibility=1, eta=1.0, rank_tol=1e-8,
                                     seed=1234, construct="device")
    h.sync()
    h.keep_original()
    h.set_gemm_tile(128)
    h.set_precision(pp.BF16 if args.form == "bf16" else pp.FP64)
    b = torch.from_numpy(pp.rhs(n, 8)).cuda()
    x = torch.empty_like(b)
    for which, nrhs in ((0, 1), (1, 8)):
        tasks, _, _, _ = h.encode_program(which, nrhs, [0] * 5)
        ef, et, _ = h.edges(which, nrhs)
        h.enable_trace(which, nrhs)
        for _ in range(2):
            if which == 0:
                h.restore()
                h.factor()
            else:
                h.solve(b, x)
            h.sync()
        tr = h.read_trace(which, nrhs)
        analyse(f"{'factor' if which == 0 else 'solve, 8 RHS'} of the 3-D Laplace job, N = {n}, {args.form} form",
                tasks, tr, ef, et)


def time_gmres(pp, ctx, torch, args):
    """Per-component device times of one GMRES step over the uneven batch (512 instances, N
    log-uniform in [1024, 16384], exp(-r/0.1) + 1e-2 I on U[0,1]^2, weak admissibility, leaf
    128, rank <= 24 at 1e-7, built on the device): the merged solve, the batched product in FP64
    and with FP32-evaluated entries, the last Arnoldi launch of a cycle, one whole cycle, and the
    merged factor (CUDA events on the batch's stream, best of 3)."""
    rng = np.random.default_rng(4096)
    s = torch.cuda.Stream()
    hs, probs = [], []
    with torch.cuda.stream(s):
        for i in range(args.instances):
            n = int(round(np.exp(rng.uniform(np.log(1024), np.log(16384))) / 64)) * 64
            h, prob = pp.make_kernel_problem(ctx, n, 2, "exp", 0.1, 128, 24, shift=1e-2, seed=4096 + 31 * i,
                                             rank_tol=1e-7, construct="device", stream=s)
            h.keep_original(s)
            hs.append(h)
            probs.append(prob)
    s.synchronize()
    batch = pp.Batch(ctx, hs)
    batch.autotune(s)
    bs = [torch.from_numpy(pp.rhs(p.n, 1, seed=3 + i)).cuda() for i, p in enumerate(probs)]
    gm = pp.BatchGMRES(batch, probs, m=args.restart, stream=s, lowp=True)

    def timeit(fn, reps=3):
        best = float("inf")
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s):
                a.record(s)
                fn()
                b.record(s)
            b.synchronize()
            best = min(best, a.elapsed_time(b))
        return best

    with torch.cuda.stream(s):
        batch.factor(s)
        gm.reset(bs)
        gm.cycle(bs)
    s.synchronize()
    v0 = [V[0].view(-1, 1) for V in gm.V]
    z0 = [Z[0].view(-1, 1) for Z in gm.Z]
    prod = [(p.kernel, p.p0, p.shift, pts, z, None, gm.zero[:p.n], V[1].view(-1, 1))
            for p, pts, z, V in zip(probs, gm.pts, z0, gm.V)]
    L = pp.lib()
    res = {
        "instances": len(probs), "n_total": int(sum(p.n for p in probs)),
        "kernel_evaluations_per_product": float(sum(p.n * (p.n + 1) / 2 for p in probs)),
        "merged_solve_ms": timeit(lambda: batch.solve(v0, z0, s)),
        "product_fp64_ms": timeit(lambda: ctx.kernel_residual_batch(prod, s)),
        "product_fp32_entries_ms": timeit(lambda: ctx.kernel_residual_batch(prod, s, lowp=True)),
        "arnoldi_last_step_ms": timeit(lambda: L.pp_gmres_arnoldi(gm._h, args.restart - 1, pp._stream_handle(s))),
        "cycle_ms": timeit(lambda: gm.cycle(bs), 1),
        "restore_and_factor_ms": timeit(lambda: (batch.restore(s), batch.factor(s)), 1),
    }
    for k, v in res.items():
        print(f"{k:32s} {v:.6g}" if isinstance(v, float) else f"{k:32s} {v}")


def time_dag(pp, torch, args):
    """DAG build of the mixed configuration's factor program (3-D Laplace, leaf 512, eta 1,
    rank <= 32, BF16 form) on the host and on the device: the program's tasks and edges, the
    DAG build's wall time, the whole program build's."""
    import time
    n = args.n if args.n != 8192 else 65536
    rng = np.random.default_rng(1234)
    pts = rng.uniform(0, 1, (n, 3))
    pts = pts[pp.morton_order(pts)]
    for mode in ("host", "device"):
        ctx = pp.Context(device=0)
        if mode == "device":
            ctx.set_device_dag(True)
        h = pp.Hierarchical.geometric(ctx, pts, 512, 1, 1.0, 32)
        h.set_rank_tolerance(1e-8)
        h.set_precision(pp.BF16)
        t0 = time.perf_counter()
        info = h.program_info(0)
        wall = time.perf_counter() - t0
        ms, on_dev = h.dag_info(0)
        print(f"{mode:6s} tasks {info['n_tasks']} edges {info['n_edges']} dag {ms:.1f} ms (on device: {on_dev}) "
              f"program build {info['host_build_ms']:.1f} ms (wall {1e3 * wall:.1f} ms)")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=8192)
    ap.add_argument("--leaf", type=int, default=256)
    ap.add_argument("--rank", type=int, default=16)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--gemm-tile", type=int, default=128, help="output tile edge of the factor's products")
    ap.add_argument("--out", default=None, help="also save the raw trace (npz)")
    ap.add_argument("--workload", default="hodlr", choices=["hodlr", "laplace3d", "gmres", "dag"])
    ap.add_argument("--instances", type=int, default=512, help="gmres: instances of the uneven batch")
    ap.add_argument("--restart", type=int, default=32, help="gmres: restart length")
    ap.add_argument("--form", default="bf16", choices=["bf16", "fp64"])
    args = ap.parse_args()
    import torch

    pp = _load()
    ctx = pp.Context(device=0)
    if args.workload == "laplace3d":
        trace_laplace3d(pp, ctx, torch, args)
        return
    if args.workload == "gmres":
        time_gmres(pp, ctx, torch, args)
        return
    if args.workload == "dag":
        time_dag(pp, torch, args)
        return
    h, prob = pp.make_kernel_problem(ctx, args.n, 2, "inv", 1e-3, args.leaf, args.rank, seed=1234)
    h.set_gemm_tile(args.gemm_tile)
    h.upload()
    h.keep_original()
    raw = {}
    for which in (0, 1):
        tasks, _, _, _ = h.encode_program(which, 1, [0] * 5)
        ef, et, _ = h.edges(which, 1)
        raw[f"tasks{which}"], raw[f"ef{which}"], raw[f"et{which}"] = tasks, ef, et
    b = torch.from_numpy(pp.rhs(args.n)).cuda()
    x = torch.empty_like(b)
    h.enable_trace(0)
    h.enable_trace(1, 1)
    for _ in range(3):
        h.restore()
        h.factor()
        h.solve(b, x)
        h.sync()
    raw["tr0"], raw["tr1"] = h.read_trace(0), h.read_trace(1, 1)
    analyse("factor, one job", raw["tasks0"], raw["tr0"], raw["ef0"], raw["et0"])
    analyse("solve, one job", raw["tasks1"], raw["tr1"], raw["ef1"], raw["et1"])
    if args.batch > 1:
        hs = [h] + [pp.Hierarchical.geometric(ctx, prob.points, args.leaf, 0, 1.0, args.rank)
                    for _ in range(args.batch - 1)]
        for q in hs[1:]:
            q.set_gemm_tile(args.gemm_tile)
            q.host_arena()[:] = h.host_arena()
            q.upload()
            q.keep_original()
        bt = pp.Batch(ctx, hs)
        bt.enable_trace(0)
        bt.enable_trace(1, 1)
        bs = [torch.from_numpy(pp.rhs(args.n, 1, seed=7 + i)).cuda() for i in range(args.batch)]
        xs = [torch.empty_like(q) for q in bs]
        for _ in range(3):
            bt.restore()
            bt.factor()
            bt.solve(bs, xs)
            bt.sync()
        for which, name in ((0, "factor"), (1, "solve")):
            tr = bt.read_trace(which, 1).astype(np.int64)
            raw[f"btr{which}"] = tr
            dur = tr[:, 1] - tr[:, 0]
            mk = tr[:, 1].max() - tr[:, 0].min()
            print(f"== batched {name}, {args.batch} jobs: tasks {len(tr)} makespan {mk / 1e3:.1f} us, "
                  f"busy {dur.sum() / 1e3:.0f} us, average parallelism {dur.sum() / mk:.1f}")
    if args.out:
        np.savez_compressed(args.out, **raw)


if __name__ == "__main__":
    main()
