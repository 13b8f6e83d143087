"""Benchmark: FP64-accurate TFLOP/s (2mnk/t) of ca3dmm_engine_exec on one B200.

Workload (N=1): square FP64 GEMM M=N=K=8000, transA=0, transB=0, the
reference's 24-rank virtual grid 4x2x3 (cuboid 2000x4000x2667), entries
sign*(1+u)*2^e with e uniform in [-8,8] (seeded hash).  A step is one
ca3dmm_engine_exec over device-resident A and B (512 MB each, larger than
L2, so no flush is needed).  Three legs are measured, each with its error
against the double-double oracle on sampled entries: plain FP64 (DMMA), split
precision by INT8 slices (7 slices) and split precision by the modular scheme
(one INT8 GEMM per modulus, the count the engine chooses for this k).  The
headline is the fastest split leg whose error is no worse than the plain
leg's.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With torchrun (N>1) every rank runs an independent replica ("replicas only":
the path has no data-path collective on one node in this scope) and the
reported value is the sum over ranks of the work divided by the max time.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M = N = K = 8000
P = 24
GRID = (4, 2, 3)
METRIC = "FP64-accurate TFLOP/s (2mnk/t): split-precision vs plain DMMA, equal error"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--trans-a", type=int, default=0)
    ap.add_argument("--trans-b", type=int, default=0)
    ap.add_argument("--size", type=int, default=M)
    ap.add_argument("--p", type=int, default=P, help="virtual ranks of the square workload")
    ap.add_argument("--grid", default="%dx%dx%d" % GRID,
                    help="virtual grid mp x np x kp of the square workload, or auto (the "
                         "reference's own choice for --p ranks)")
    ap.add_argument("--dist", default="signed_exp", choices=["signed_exp", "uniform"],
                    help="square workload entries: sign*(1+u)*2^e, e in [-8,8] (8000^3), or "
                         "uniform in [-1,1) (the 2048^3 example workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--gemm", default="auto", choices=["auto", "plain", "ozaki", "crt"],
                    help="leg timed as the headline (auto: the fastest split leg whose error is "
                         "no worse than plain's); a fixed leg keeps profiling captures on one path")
    ap.add_argument("--workload", default="square", choices=["square", "grouped", "btb"],
                    help="square: the headline 8000^3 engine exec; grouped: 256 uneven "
                         "independent GEMMs in one graph-captured launch; btb: B^T B of a "
                         "1048576 x 512 B on a 1x1x32 grid")
    ap.add_argument("--nprob", type=int, default=256)
    ap.add_argument("--btb-rows", type=int, default=1048576,
                    help="rows of B for --workload btb (smaller values: profiling captures)")
    ap.add_argument("--no-slice-sweep", action="store_true",
                    help="skip timing the other split-precision slice counts")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="also time the reference's own GPU path (cuBLAS DGEMM, MPI steps staged "
                         "through host memory) on this GPU, for context")
    ap.add_argument("--ref-gpu-child", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--sharded", action="store_true",
                    help="square workload as one CA3DMM across the launched GPUs (one rank per "
                         "GPU on the reference's grid for p = N, NCCL all-to-alls; strong "
                         "scaling) instead of N independent replicas")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region: samples
    every 100 ms in a reader thread; mark() brackets the timed region and only
    the samples read between the marks are summarised."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def mark(self):
        return len(self.samples)

    def stop(self, i0=0, i1=None):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        window = self.samples[i0:i1] if i1 is not None and i1 > i0 else self.samples[i0:i0 + 1]
        sm = [float(s[1]) for s in window if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in window if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in window:
            for nm, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(window)}


def max_over_ranks(ms, world, device="cuda"):
    """The slowest rank's time: every rank contributes its own device-timed ms."""
    if world == 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_tflops(flops_per_rank, world, ms):
    """Whole-job throughput: the work of all ranks over the slowest rank's time."""
    return world * flops_per_rank / (ms * 1e-3) / 1e12


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def ncu_traffic():
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "ncu_traffic.json")))
    except Exception:
        return {}


def make_inputs(n, trans_a, dist="signed_exp"):
    from oracle import oracle as orc
    if dist == "uniform":
        return orc.gen_uniform(1, n, n), orc.gen_uniform(2, n, n)
    A = orc.gen_signed_exp(101, n, n)
    B = orc.gen_signed_exp(202, n, n)
    return A, B


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def grid_of(args):
    """The square workload's virtual grid: a tuple, or None for the planner's choice."""
    if args.grid == "auto":
        return None
    g = tuple(int(x) for x in args.grid.lower().split("x"))
    if len(g) != 3:
        raise SystemExit("--grid wants mp x np x kp, e.g. 4x2x3, or auto")
    return g


def grid_str(grid):
    return "auto" if grid is None else "%dx%dx%d" % tuple(grid)


def ref_cpu_run(A, B, ta, n, ntest, tb=0, p=P, grid=GRID, matmul=False):
    """The reference's own CPU path (src/ca3dmm.c, DEV_TYPE_HOST, OpenBLAS),
    compiled unmodified under the thread-backed MPI subset: p rank threads
    with one BLAS thread each, driven as examples/example_AB.c drives it (one
    warm-up exec, then `ntest` timed execs).  Returns exec ms per timed exec
    of rank 0 (with matmul: also its "matmul only" ms, examples/example_AB.c:190),
    or None when the reference build is absent."""
    from oracle import oracle as orc
    if orc.ref_lib() is None:
        return None
    _, times, _, g = orc.ref_ca3dmm(p, n, n, n, ta, tb, A, B, grid=grid, ntest=ntest, timeout=600.0)
    if matmul:
        return list(times[:, 0]), list(times[:, 1]), g
    return list(times[:, 0])


def cpu_baseline(A, B, ta, n, budget_s=20.0, tb=0, p=P, grid=GRID):
    """CPU baseline on this host: the reference's own CPU path when it was
    built (kind "reference"), else the oracle's numpy restatement of the
    virtual-rank algorithm on k-slab 0 (kind "port")."""
    from oracle import oracle as orc
    flops = 2.0 * n * n * n
    r = ref_cpu_run(A, B, ta, n, 1, tb, p=p, grid=grid, matmul=True)
    if r is not None:
        ms, mm, _ = r
        out = {"value": flops / (ms[0] * 1e-3) / 1e12, "unit": "TFLOP/s",
               "cores": min(p, cpu_cores()), "kind": "reference",
               "sample": "one full %d^3 exec (after one warm-up) of the reference's CPU path, "
                         "%d rank threads on grid %s, 1 OpenBLAS thread per rank"
                         % (n, p, grid_str(grid)),
               "matmul_only_value": flops / (mm[0] * 1e-3) / 1e12}
        # the second protocol of the study: one rank per host core, the
        # reference's own grid choice for that many ranks
        pc = cpu_cores()
        if pc != p:
            r2 = ref_cpu_run(A, B, ta, n, 1, tb, p=pc, grid=None, matmul=True)
            if r2 is not None:
                ms2, mm2, g2 = r2
                out["p_equals_cores"] = {
                    "p": pc, "grid": "%dx%dx%d" % g2[:3],
                    "value": flops / (ms2[0] * 1e-3) / 1e12,
                    "matmul_only_value": flops / (mm2[0] * 1e-3) / 1e12}
        return out
    cores = os.cpu_count()
    try:
        from threadpoolctl import threadpool_info
        cores = max([i.get("num_threads", 0) for i in threadpool_info()] + [1])
    except Exception:
        pass
    k0, kz = orc.block_spos_size(n, 3, 0)
    Ask = np.asfortranarray((A.T if ta else A)[:, k0:k0 + kz])
    Bsk = np.asfortranarray((B.T if tb else B)[k0:k0 + kz, :])
    reps, t = 0, 0.0
    while True:
        t0 = time.perf_counter()
        orc.cpu_ca3dmm(Ask, Bsk, 0, 0, n, n, kz, 4, 2, 1)
        t += time.perf_counter() - t0
        reps += 1
        if t > budget_s / 4 or reps >= 3:
            break
    flops = 2.0 * n * n * kz * reps
    return {"value": flops / t / 1e12, "unit": "TFLOP/s", "cores": cores, "kind": "port",
            "sample": "k-slab 0 of the 4x2x3 grid (8 rank cuboids, %dx%dx%d), %d rep(s), "
                      "numpy/OpenBLAS local GEMMs + slab sum" % (n, n, kz, reps)}


def reference_arm(args, world, rank):
    """The reference's CPU implementation of the path on this host's cores
    (rank 0 only): each step is one full ca3dmm_engine_exec of the reference
    over the same 8000^3 inputs and 4x2x3 grid."""
    if rank != 0:
        return
    n = args.size
    A, B = make_inputs(n, args.trans_a, args.dist)
    steps, warm = max(args.steps, 1), max(args.warmup, 0)
    flops = 2.0 * n * n * n
    grid = grid_of(args)
    ms = ref_cpu_run(A, B, args.trans_a, n, warm + steps, args.trans_b, p=args.p, grid=grid)
    if ms is not None:
        t = float(np.mean(ms[warm:]))
        v = flops / (t * 1e-3) / 1e12
        base = {"value": v, "unit": "TFLOP/s", "cores": min(args.p, cpu_cores()),
                "kind": "reference",
                "sample": "%d full %d^3 execs of the reference's CPU path (%d rank threads, grid "
                          "%s, 1 OpenBLAS thread per rank) after %d warm-up"
                          % (steps, n, args.p, grid_str(grid), warm + 1)}
        note = ("reference src/ca3dmm.c CPU path (DEV_TYPE_HOST, OpenBLAS 0.3.31) compiled "
                "unmodified; MPI ranks are threads of one process")
    else:
        vals = []
        for _ in range(warm):
            cpu_baseline(A, B, args.trans_a, n, budget_s=4.0, tb=args.trans_b, p=args.p, grid=grid)
        for _ in range(steps):
            base = cpu_baseline(A, B, args.trans_a, n, budget_s=4.0, tb=args.trans_b, p=args.p,
                                grid=grid)
            vals.append(base["value"])
        v = float(np.median(vals))
        base["value"] = v
        t = flops / (v * 1e12) * 1e3
        note = "reference build absent: the oracle's restatement of its CPU path"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "TFLOP/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": warm, "ms_per_step": t,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": square_desc(n, args.trans_a, args.trans_b, args.p, grid,
                                               args.dist),
                       "l2": square_l2(n)},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": note}
    print(json.dumps(line), flush=True)


def grouped_problems(nprob, seed=2024):
    """256 GEMMs, m, n, k = round(exp(U[ln 64, ln 4096])), random trans flags,
    entries u * 2^e with u uniform in [-1, 1), e uniform in [-4, 4]."""
    rng = np.random.default_rng(seed)
    dims = np.exp(rng.uniform(np.log(64), np.log(4096), size=(nprob, 3))).round().astype(int)
    ta = rng.integers(0, 2, nprob)
    tb = rng.integers(0, 2, nprob)
    return [(int(m), int(n), int(k), int(ta[i]), int(tb[i])) for i, (m, n, k) in enumerate(dims)]


def run_grouped(args, world, rank, local):
    """256 uneven GEMMs: one persistent grouped launch (captured in a CUDA graph)
    against one plain DMMA launch per GEMM.  With N ranks each GPU runs its own
    replica of the batch (weak scaling): the time is the slowest rank's and the
    value counts every rank's flops."""
    import torch
    import ca3dmm_b200 as cb
    from oracle import oracle as orc
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    probs = grouped_problems(args.nprob)
    flops = sum(2.0 * m * n * k for m, n, k, _, _ in probs)
    dA, dB, dC, lda, ldb, ldc = [], [], [], [], [], []
    for i, (m, n, k, ta, tb) in enumerate(probs):
        A = orc.gen_signed_exp(3000 + i, *((k, m) if ta else (m, k)), emin=-4, emax=4, unit=True)
        B = orc.gen_signed_exp(4000 + i, *((n, k) if tb else (k, n)), emin=-4, emax=4, unit=True)
        dA.append(torch.from_numpy(A.ravel(order="F").copy()).cuda()); lda.append(A.shape[0])
        dB.append(torch.from_numpy(B.ravel(order="F").copy()).cuda()); ldb.append(B.shape[0])
        dC.append(torch.zeros(m * n, dtype=torch.float64, device="cuda")); ldc.append(m)
    stream = torch.cuda.Stream()
    res = {}

    def timed(fn, steps):
        # everything (library launches, graph replays, events) on `stream`
        with torch.cuda.stream(stream):
            for _ in range(max(args.warmup, 1)):
                fn()
            torch.cuda.synchronize()
            if world > 1:
                torch.distributed.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                fn()
            e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        return max_over_ranks(e0.elapsed_time(e1) / steps, world)

    # one plain DMMA launch (pack + GEMM) per product
    singles = [cb.GroupedGemm([m], [n], [k], [ta], [tb]) for m, n, k, ta, tb in probs]
    for i, g in enumerate(singles):
        g.set_stream(stream.cuda_stream, 0)

    def run_singles():
        for i, g in enumerate(singles):
            g.exec([dA[i]], [lda[i]], [dB[i]], [ldb[i]], [dC[i]], [ldc[i]])
    res["per_gemm_launches_ms"] = timed(run_singles, args.steps)
    for mode, sl, key in ((cb.GEMM_PLAIN, 0, "grouped_plain"), (cb.GEMM_OZAKI, 7, "grouped_ozaki7"),
                          (cb.GEMM_CRT, 0, "grouped_crt")):
        g = cb.GroupedGemm([p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs],
                           [p[3] for p in probs], [p[4] for p in probs], mode=mode, slices=sl)
        assert g.ok
        assert g.exec(dA, lda, dB, ldb, dC, ldc) == 0
        g.set_stream(stream.cuda_stream, 0)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            g.exec(dA, lda, dB, ldb, dC, ldc)
        res[key + "_ms"] = timed(graph.replay, args.steps)
        del graph
    # the headline: the faster split-precision leg (both at least as accurate as
    # plain FP64 on these entries)
    head = min(("grouped_ozaki7_ms", "grouped_crt_ms"), key=lambda x: res[x])
    v = whole_job_tflops(flops, world, res[head])
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    out = {"metric": METRIC, "value": v, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": res[head], "gemm": head.replace("_ms", ""),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic",
           "config": {"workload": "%d independent GEMMs, m,n,k log-uniform in [64,4096], random "
                                  "trans, one grouped launch in a CUDA graph" % len(probs),
                      "total_flop": flops},
           "legs_ms": res,
           "legs_tflops": {k.replace("_ms", ""): whole_job_tflops(flops, world, t)
                           for k, t in res.items()}}
    print(json.dumps(out), flush=True)


BTB_N, BTB_P, BTB_GRID = 512, 32, (1, 1, 32)


def make_btb(k, n, seed=303):
    """B (k x n, column-major) with column j ~ N(0, 1) * 10^u_j, u_j uniform in
    [-3, 3], from a seeded torch generator (the tall-skinny Gram workload)."""
    import torch
    g = torch.Generator().manual_seed(seed)
    z = torch.randn(n, k, dtype=torch.float64, generator=g)
    u = torch.rand(n, dtype=torch.float64, generator=g) * 6.0 - 3.0
    z.mul_(torch.pow(10.0, u)[:, None])
    return z.numpy().T          # Fortran-ordered view of the (n, k) row-major buffer


def square_desc(n, ta, tb, p=P, grid=GRID, dist="signed_exp"):
    """The square workload's name, the same in both arms' JSON lines."""
    cub = " (cuboid 2000x4000x2667 at 8000^3)" if (p, grid) == (P, GRID) else ""
    ent = "uniform in [-1,1)" if dist == "uniform" else "sign*(1+u)*2^e, e in [-8,8]"
    return ("ca3dmm_exec M=N=K=%d transA=%d transB=%d, %d virtual ranks, grid %s%s, entries %s"
            % (n, ta, tb, p, grid_str(grid), cub, ent))


def square_l2(n):
    """The L2 note of the square workload, the same in both arms' JSON lines."""
    mb = n * n * 8 / 1e6
    return ("inputs larger than L2 (%.0f MB per operand), no flush" % mb if n * n * 8 > 126e6
            else "inputs of %.1f MB per operand (smaller than L2), no flush" % mb)


def workload(args):
    if args.workload == "btb":
        rows = args.btb_rows
        B = make_btb(rows, BTB_N)
        return {"m": BTB_N, "n": BTB_N, "k": rows, "ta": 0, "tb": 0, "btb": True, "p": BTB_P,
                "grid": BTB_GRID, "A": None, "B": B,
                "label": "btb %dx%d grid 1x1x32" % (rows, BTB_N),
                "desc": "ca3dmm_exec B^T B, B %dx%d, columns N(0,1)*10^u, u in [-3,3], 32 virtual "
                        "ranks on grid 1x1x32 (kp-slab reduction on device)" % (rows, BTB_N),
                "l2": "B is %.1f GB%s, no flush" % (rows * BTB_N * 8 / 1e9,
                                                    ", larger than L2" if rows * BTB_N * 8 > 126e6
                                                    else "")}
    n = args.size
    A, B = make_inputs(n, args.trans_a, args.dist)
    grid = grid_of(args)
    return {"m": n, "n": n, "k": n, "ta": args.trans_a, "tb": args.trans_b, "btb": False,
            "p": args.p, "grid": grid,
            "A": A, "B": B, "label": "square %d^3 grid %s" % (n, grid_str(grid)),
            "desc": square_desc(n, args.trans_a, args.trans_b, args.p, grid, args.dist),
            "l2": square_l2(n)}


def sampled_error(Cdev, wl, nsample=2048):
    """Errors of sampled device entries against the double-double oracle."""
    import torch
    from oracle import oracle as orc
    m, n, k = wl["m"], wl["n"], wl["k"]
    if wl["btb"]:
        ii, jj = orc.sample_indices(n, n, nrand=256, nlines=0)
        hi, lo, ab = orc.dd_entries(wl["B"], wl["B"], 1, 0, k, ii, jj)
    else:
        ii, jj = orc.sample_indices(m, n, nrand=nsample, nlines=1)
        hi, lo, ab = orc.dd_entries(wl["A"], wl["B"], wl["ta"], wl["tb"], k, ii, jj)
    idx = torch.from_numpy(ii + jj * m).cuda()
    return orc.errors(Cdev[idx].cpu().numpy(), hi, lo, ab)


def btb_cpu_baseline(wl, rows=131072):
    """The reference's CPU B^T B on the first `rows` rows of B (same 32-rank
    1x1x32 grid, one warm-up and one timed exec)."""
    from oracle import oracle as orc
    if orc.ref_lib() is None:
        return None
    n = wl["n"]
    Bs = np.asfortranarray(wl["B"][:rows, :])
    _, times, _, _ = orc.ref_ca3dmm(BTB_P, n, n, rows, 0, 0, None, Bs, grid=BTB_GRID, ntest=1,
                                   btb=True, timeout=600.0)
    return {"value": 2.0 * n * n * rows / (times[0, 0] * 1e-3) / 1e12, "unit": "TFLOP/s",
            "cores": min(BTB_P, cpu_cores()), "kind": "reference",
            "sample": "B^T B of the first %d of %d rows, reference CPU path, 32 rank threads on "
                      "grid 1x1x32" % (rows, wl["k"])}


def ref_gpu_child(args):
    """Runs in a child process (its own CUDA runtime, and the reference's
    exit-on-error paths stay out of the bench): the reference's GPU path over
    the same workload, on the workload's grid and on one rank (where the
    reference's "matmul only" time is one cuBLAS DGEMM of the whole product)."""
    from oracle import oracle as orc
    wl = workload(args)
    m, n, k = wl["m"], wl["n"], wl["k"]
    flops = 2.0 * m * n * k
    out = {}
    for name, p, grid in (("grid", wl["p"], wl["grid"]), ("one_rank", 1, None)):
        if name == "one_rank" and wl["btb"]:
            continue
        t0 = time.perf_counter()
        _, times, g = orc.ref_ca3dmm_cuda(p, m, n, k, wl["ta"], wl["tb"], wl["A"], wl["B"],
                                          grid=grid, ntest=3, btb=wl["btb"], timeout=600.0)
        ex, mm = float(np.median(times[:, 0])), float(np.median(times[:, 1]))
        out[name] = {"p": p, "grid": "%dx%dx%d" % g[:3], "exec_ms": ex, "matmul_only_ms": mm,
                     "value": flops / (ex * 1e-3) / 1e12,
                     "matmul_only_value": flops / (mm * 1e-3) / 1e12,
                     "wall_s": time.perf_counter() - t0}
    print("REFGPU " + json.dumps(out), flush=True)


def ref_gpu_leg(args):
    """The reference's own GPU path on this GPU (context only): oracle/_ref's
    build of src/*.c with USE_CUDA and src/cuda_proxy.cu for sm_100a, p rank
    threads sharing the GPU, cuBLAS calls serialised.  None when not built."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_ca3dmm_cuda.so")):
        return None
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--ref-gpu-child"] + \
        [a for a in sys.argv[1:] if a != "--ref-gpu"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    for line in r.stdout.splitlines():
        if line.startswith("REFGPU "):
            res = json.loads(line[7:])
            res["unit"] = "TFLOP/s"
            res["note"] = ("the reference's GPU path (DEV_TYPE_CUDA: cuBLAS DGEMM per Cannon step, "
                           "redistribution, allgather and kp reduction staged through pinned host "
                           "memory) on this GPU, 3 timed execs after one warm-up, median; context, "
                           "not the reference arm")
            return res
    return {"unavailable": "reference GPU run failed (rc %d): %s" %
            (r.returncode, (r.stderr or r.stdout).strip().splitlines()[-1:])}


def run_sharded(args, world, rank, local):
    """CA3DMM across the launched GPUs (the C engine of include/ca3dmm_dist.h through
    ca3dmm_b200.dist, over NCCL): A, B and C
    of the square workload in examples/example_AB.c's 1D column blocks, one rank
    per GPU on the reference's grid for p = N (or --grid when its product is at
    most N).  Total work is fixed (strong scaling); time is the slowest rank's."""
    import datetime
    import torch
    import torch.distributed as dist
    import ca3dmm_b200 as cb
    from ca3dmm_b200.dist import DistCa3dmmEngine
    from oracle import oracle as orc
    torch.cuda.set_device(local)
    if world == 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if "MASTER_PORT" not in os.environ:
            import socket
            with socket.socket() as sk:
                sk.bind(("127.0.0.1", 0))
                os.environ["MASTER_PORT"] = str(sk.getsockname()[1])
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    n, ta, tb = args.size, args.trans_a, args.trans_b
    grid = grid_of(args)
    if grid is not None and grid[0] * grid[1] * grid[2] > world:
        grid = None
    A, B = make_inputs(n, ta, args.dist)
    s0, sz = cb.calc_block_spos_size(n, world, rank)
    blk = (0, n, s0, sz)

    def cols(X):
        return torch.from_numpy(np.asfortranarray(X[:, s0:s0 + sz]).ravel(order="F").copy()
                                if sz else np.zeros(1)).cuda()

    dA, dB = cols(A), cols(B)
    dC = torch.zeros(max(n * sz, 1), dtype=torch.float64, device="cuda")
    oz_slices = int(os.environ.get("CA3DMM_BENCH_SLICES", "7"))
    legs = {}
    flops = 2.0 * n * n * n
    for mode, key, sl in ((cb.GEMM_PLAIN, "plain", 0), (cb.GEMM_OZAKI, "ozaki", oz_slices),
                          (cb.GEMM_CRT, "crt", 0)):
        e = DistCa3dmmEngine(n, n, n, ta, tb, blk, blk, blk, proc_grid=grid, gemm_mode=mode,
                             slices=sl)
        for _ in range(args.warmup):
            e.exec(dA, n, dB, n, dC, n)
        e.reset_stat()
        dist.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(args.steps):
            e.exec(dA, n, dB, n, dC, n)
        ev1.record()
        torch.cuda.synchronize()
        ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world)
        st = {kk: (v / max(e.stats["n_exec"], 1) if kk != "n_exec" else v)
              for kk, v in e.stats.items()}
        # this rank's C columns against the double-double truth (sampled)
        err = None
        if sz:
            ii, jj = orc.sample_indices(n, sz, nrand=512, nlines=0)
            hi, lo, ab = orc.dd_entries(A, B, ta, tb, n, ii, jj + s0)
            err = orc.errors(dC[torch.from_numpy(ii + jj * n).cuda()].cpu().numpy(), hi, lo, ab)
        legs[key] = {"ms_per_step": ms, "tflops": flops / (ms * 1e-3) / 1e12,
                     "grid": "%dx%dx%d" % (e.mp, e.np_, e.kp), "idle_ranks": e.rp,
                     "rank0_phases_ms": st, "rank0_err": err}
        e.free()
    # the headline: the faster split-precision leg whose rank-0 errors are no
    # worse than the plain leg's (the same rule as the single-GPU bench)
    ep = legs["plain"]["rank0_err"]
    head = "ozaki"
    ec = legs["crt"]["rank0_err"]
    if ep is None or ec is None or (ec["normwise"] <= ep["normwise"] and
                                    ec["vs_absprod"] <= ep["vs_absprod"]):
        if legs["crt"]["ms_per_step"] < legs["ozaki"]["ms_per_step"]:
            head = "crt"
    out = {"metric": METRIC, "value": legs[head]["tflops"], "unit": "TFLOP/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": legs[head]["ms_per_step"],
           "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic",
           "gemm": head,
           "config": {"workload": "sharded " + square_desc(n, ta, tb, world, None, args.dist)
                      .replace("virtual ranks", "GPU ranks"),
                      "layout": "A, B, C in 1D column blocks over the ranks",
                      "exchange": "the C engine (ca3dmm_dist_engine_*) over NCCL "
                                  "all_to_all_single: operand panels, C pieces",
                      "l2": "inputs larger than L2 at 8000^3, no flush"},
           "legs": legs}
    if rank == 0:
        print(json.dumps(out), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def main():
    args = parse()
    if args.sharded and args.impl == "ours":
        world, rank, local = dist_setup(args)
        run_sharded(args, world, rank, local)
        return
    if args.ref_gpu_child:
        ref_gpu_child(args)
        return
    world, rank, local = dist_setup(args)
    if args.workload == "grouped" and args.impl == "ours":
        run_grouped(args, world, rank, local)
        return
    if args.impl == "reference":
        reference_arm(args, world, rank)
        return
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import ca3dmm_b200 as cb
    wl = workload(args)
    m, n, k, ta, btb = wl["m"], wl["n"], wl["k"], wl["ta"], wl["btb"]
    lda = (k if ta else m) if not btb else 0
    ldb = k
    hA = None if btb else torch.from_numpy(wl["A"].ravel(order="F")).pin_memory()
    hB = torch.from_numpy(wl["B"].ravel(order="F")).pin_memory()
    dA = None if btb else hA.cuda()
    dB = hB.cuda()
    dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.default_stream()
    flops = 2.0 * m * n * k

    def engine():
        return cb.Ca3dmmEngine(m, n, k, ta, wl["tb"], p=wl["p"], proc_grid=wl["grid"], btb=btb)

    def leg(eng, steps, warmup):
        for _ in range(warmup):
            if eng.exec(dA, lda, dB, ldb, dC, m):
                raise RuntimeError("exec failed")
        torch.cuda.synchronize()
        eng.reset_stat()
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        # the engine runs synchronously on the legacy default stream; events on it
        evs[0].record(stream)
        for i in range(steps):
            eng.exec(dA, lda, dB, ldb, dC, m)
            evs[i + 1].record(stream)
        torch.cuda.synchronize()
        st = eng.s
        per = [evs[i].elapsed_time(evs[i + 1]) for i in range(steps)]
        return {"ms_per_step": evs[0].elapsed_time(evs[-1]) / steps,
                "ms_median": float(np.median(per)), "ms_min": float(min(per)),
                "gemm_ms": st.cannon_ms / max(st.n_exec, 1),
                "pack_ms": st.redist_ms / max(st.n_exec, 1),
                "reduce_ms": st.reduce_ms / max(st.n_exec, 1)}

    legs = {}
    eng_plain = engine()
    assert eng_plain.ok, "engine init failed"
    eng_plain.set_gemm_mode(cb.GEMM_PLAIN)
    oz_slices = int(os.environ.get("CA3DMM_BENCH_SLICES", "7"))
    crt_moduli = int(os.environ.get("CA3DMM_BENCH_MODULI", "0"))   # 0: the engine's choice
    eng_oz = engine()
    if not (eng_oz.ok and eng_oz.set_gemm_mode(cb.GEMM_OZAKI, oz_slices) == 0 and
            eng_oz.exec(dA, lda, dB, ldb, dC, m) == 0):
        raise RuntimeError("split-precision engine failed")
    eng_crt = engine()
    if not (eng_crt.ok and eng_crt.set_gemm_mode(cb.GEMM_CRT, crt_moduli) == 0 and
            eng_crt.exec(dA, lda, dB, ldb, dC, m) == 0):
        raise RuntimeError("modular split-precision engine failed")
    engines = {"plain": eng_plain, "ozaki": eng_oz, "crt": eng_crt}
    legs["plain"] = leg(eng_plain, 1, args.warmup)
    legs["plain"]["err"] = sampled_error(dC, wl)
    legs["ozaki"] = leg(eng_oz, 1, args.warmup)
    legs["ozaki"]["err"] = sampled_error(dC, wl)
    legs["ozaki"]["slices"] = oz_slices
    legs["crt"] = leg(eng_crt, 1, args.warmup)
    legs["crt"]["err"] = sampled_error(dC, wl)
    legs["crt"]["moduli"] = eng_crt.s.crt_moduli
    legs["crt"]["bits"] = eng_crt.s.crt_bits
    if not btb and not args.no_slice_sweep:
        # the other slice counts: time and error of each (one timed exec)
        sweep = {}
        for sc in (3, 4, 5, 6, 8):
            if sc == oz_slices:
                continue
            e2 = engine()
            if e2.ok and e2.set_gemm_mode(cb.GEMM_OZAKI, sc) == 0:
                r = leg(e2, 2, 1)
                r["err"] = sampled_error(dC, wl)
                r["tflops"] = flops / (r["ms_per_step"] * 1e-3) / 1e12
                sweep[str(sc)] = r
            e2.free()
        legs["ozaki_slice_sweep"] = sweep
        # the neighbouring modulus counts of the modular scheme
        msweep = {}
        for nm in sorted({max(8, eng_crt.s.crt_moduli - 1), min(18, eng_crt.s.crt_moduli + 1)}):
            e2 = engine()
            if e2.ok and e2.set_gemm_mode(cb.GEMM_CRT, nm) == 0:
                r = leg(e2, 2, 1)
                r["err"] = sampled_error(dC, wl)
                r["tflops"] = flops / (r["ms_per_step"] * 1e-3) / 1e12
                r["bits"] = e2.s.crt_bits
                msweep[str(nm)] = r
            e2.free()
        legs["crt_moduli_sweep"] = msweep
    if btb:
        # reported separately: C = B^T B is symmetric, and with
        # CA3DMM_BTB_SYMMETRIC=1 only its upper block triangle is computed and
        # the lower triangle mirrored.  The TFLOP/s beside it is the same 2mnk / t
        # convention (an equivalent rate: the work done is about half).
        symlegs = {}
        os.environ["CA3DMM_BTB_SYMMETRIC"] = "1"
        for mode, sl in ((cb.GEMM_PLAIN, 0), (cb.GEMM_OZAKI, oz_slices)):
            es = engine()
            if es.ok and (mode == cb.GEMM_PLAIN or es.set_gemm_mode(mode, sl) == 0):
                r = leg(es, max(2, args.steps // 2), 1)
                r["err"] = sampled_error(dC, wl)
                r["tflops_2mnk_equivalent"] = flops / (r["ms_per_step"] * 1e-3) / 1e12
                symlegs["plain" if mode == cb.GEMM_PLAIN else "ozaki"] = r
            es.free()
        os.environ.pop("CA3DMM_BTB_SYMMETRIC", None)
        legs["btb_symmetric"] = symlegs
    # the headline is the fastest split-precision leg whose error against the
    # double-double truth is no worse than the plain FP64 leg's (normwise and
    # relative to |A||B|); plain FP64 when neither is
    ep = legs["plain"]["err"]
    head = "plain"
    for cand in ("ozaki", "crt"):
        ec = legs[cand]["err"]
        if ec["normwise"] <= ep["normwise"] and ec["vs_absprod"] <= ep["vs_absprod"] and (
                head == "plain" or legs[cand]["ms_per_step"] < legs[head]["ms_per_step"]):
            head = cand
    if args.gemm != "auto":
        head = args.gemm
    eng = engines[head]

    # timed region (headline leg), clocks sampled meanwhile
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    i0 = sampler.mark()
    # the timed steps, bracketed by a barrier and a device synchronisation on
    # both sides (leg() synchronises before its first and after its last event)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = cb.kernel_launches()
    res = leg(eng, args.steps, 0)
    launches = cb.kernel_launches() - l0
    if world > 1:
        torch.distributed.barrier()
    time.sleep(0.15)                      # the sample covering the region's end
    clocks = sampler.stop(i0, sampler.mark())
    ms = max_over_ranks(res["ms_per_step"], world)
    value = whole_job_tflops(flops, world, ms)
    for other in engines:
        if other != head:
            legs[other].update(leg(engines[other], max(2, args.steps // 2), 1))
    legs[head].update(res)

    # e2e: the same exec through the C ABI with host buffers
    # (ca3dmm_engine_exec_host: page-locked A, B, C; the copies in and out are
    # pipelined with the computation inside the call).  The call is synchronous
    # and uses its own streams, so the region is timed on the host with the
    # device synchronised on both sides.
    hC = torch.empty(m * n, dtype=torch.float64).pin_memory()
    e2e_steps = max(2, min(args.steps, 5))
    lda_h = 0 if btb else wl["A"].shape[0]
    if eng.exec_host(hA, lda_h, hB, ldb, hC, m) != 0:
        raise RuntimeError("exec_host failed")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        eng.exec_host(hA, lda_h, hB, ldb, hC, m)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / e2e_steps, world)

    peaks = measured_peaks()
    traffic = ncu_traffic().get(wl["label"], {})
    gemm_ms = res["gemm_ms"]
    # the burst peak for a region the board ran at full clock, the sustained one
    # (seconds-long GEMM loop under the power cap) when the sampled clocks show
    # the cap, as the timed GEMM then ran inside a long power-capped region
    capped = "sw_power_cap" in (clocks.get("reasons") or [])
    burst = 2.0 * peaks.get("bf16_tflops", 1590.0)
    sustained = 2.0 * peaks.get("bf16_tflops_sustained", 1400.0)
    int8_peak = sustained if capped else burst
    int8_src = ("of measured: 2 x measured dense bf16 %s (dense INT8 rate is twice the bf16 rate)"
                % ("sustained, the region ran under the power cap" if capped else "burst")
                if "bf16_tflops" in peaks else "of fallback")
    if head == "crt":
        nm = eng.s.crt_moduli
        ops = flops * nm                        # one INT8 product per modulus
        roof = {"bound": "tensor", "kernel": "crt_gemm_kernel",
                "achieved": ops / (gemm_ms * 1e-3) / 1e12, "peak": int8_peak, "unit": "TFLOP/s",
                "peak_source": int8_src, "traffic": traffic.get("crt_gemm_kernel")}
    elif head == "ozaki":
        s = eng.s.ozaki_slices
        ops = flops * s * (s + 1) / 2           # INT8 ops of the slice products
        roof = {"bound": "tensor", "kernel": "oz_gemm_kernel",
                "achieved": ops / (gemm_ms * 1e-3) / 1e12, "peak": int8_peak, "unit": "TFLOP/s",
                "peak_source": int8_src, "traffic": traffic.get("oz_gemm_kernel")}
    else:
        sm_mhz = peaks.get("sm_max_mhz", 1965.0)
        peak = 148 * 128 * sm_mhz * 1e6 / 1e12
        roof = {"bound": "tensor", "kernel": "dgemm_dmma_grouped",
                "achieved": flops / (gemm_ms * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                "peak_source": "nominal FP64 DMMA rate 148 SM x 128 flop/clk x max SM clock",
                "traffic": traffic.get("dgemm_dmma_grouped")}
    roof["frac"] = roof["achieved"] / roof["peak"]
    if roof["kernel"] != "dgemm_dmma_grouped":
        roof["frac_of_burst"] = roof["achieved"] / burst
    in_bytes = (0 if dA is None else dA.numel() * 8) + dB.numel() * 8
    # the metric's comparison, split precision against plain FP64 at their
    # errors against the double-double truth, as top-level keys
    split = head if head != "plain" else "crt"
    eo, ep = legs[split]["err"], legs["plain"]["err"]
    # whole-job rates of the three legs, each over its slowest rank (every rank
    # takes these reductions in the same order)
    leg_tf = {x: whole_job_tflops(flops, world, max_over_ranks(legs[x]["ms_per_step"], world))
              for x in ("plain", "ozaki", "crt")}
    plain_tf, split_tf = leg_tf["plain"], leg_tf[split]
    out = {
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": wl["desc"], "l2": wl["l2"]},
        "gemm": head, "split_leg": split, "ozaki_slices": eng_oz.s.ozaki_slices,
        "crt_moduli": eng_crt.s.crt_moduli, "crt_bits": eng_crt.s.crt_bits,
        "plain_tflops": plain_tf, "split_tflops": split_tf,
        "ozaki_tflops": leg_tf["ozaki"], "crt_tflops": leg_tf["crt"],
        "split_over_plain": split_tf / plain_tf,
        "err_normwise_split": eo["normwise"], "err_normwise_plain": ep["normwise"],
        "err_vs_absprod_split": eo["vs_absprod"], "err_vs_absprod_plain": ep["vs_absprod"],
        "roofline": roof, "clocks": clocks,
        "e2e": {"value": whole_job_tflops(flops, world, e2e_ms), "unit": "TFLOP/s",
                "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": m * n * 8},
        "gpu_launches": int(launches),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = btb_cpu_baseline(wl) if btb else \
            cpu_baseline(wl["A"], wl["B"], ta, n, tb=wl["tb"], p=wl["p"], grid=wl["grid"])
    if rank == 0 and world == 1 and args.ref_gpu:
        out["reference_gpu"] = ref_gpu_leg(args)
    out["legs"] = legs                    # detail last (slice sweep, phase times)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
