"""Benchmark: FP64-accurate TFLOP/s (2mnk/t) of ca3dmm_engine_exec on one B200.

Workload (N=1): square FP64 GEMM M=N=K=8000, transA=0, transB=0, the
reference's 24-rank virtual grid 4x2x3 (cuboid 2000x4000x2667), entries
sign*(1+u)*2^e with e uniform in [-8,8] (seeded hash).  A step is one
ca3dmm_engine_exec over device-resident A and B (512 MB each, larger than
L2, so no flush is needed).  The headline leg is the split-precision
(Ozaki INT8 on tcgen05) GEMM when available, with the plain FP64 DMMA leg
measured beside it; both legs' errors against the double-double oracle are
measured on sampled entries.

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
METRIC = "FP64-accurate TFLOP/s (2mnk/t): split-precision vs plain DMMA, equal error"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--trans-a", type=int, default=0)
    ap.add_argument("--size", type=int, default=M)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="square", choices=["square", "grouped", "btb"],
                    help="square: the headline 8000^3 engine exec; grouped: 256 uneven "
                         "independent GEMMs in one graph-captured launch; btb: B^T B of a "
                         "1048576 x 512 B on a 1x1x32 grid")
    ap.add_argument("--nprob", type=int, default=256)
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""

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
                 "--format=csv,noheader,nounits", "-lms", "200"],
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

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for nm, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


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


def make_inputs(n, trans_a):
    from oracle import oracle as orc
    A = orc.gen_signed_exp(101, n, n)
    B = orc.gen_signed_exp(202, n, n)
    return A, B


def error_vs_dd(Cdev, A, B, ta, n, nsample=2048):
    """Sampled errors of the device result against the double-double oracle."""
    import torch
    from oracle import oracle as orc
    ii, jj = orc.sample_indices(n, n, nrand=nsample, nlines=1)
    hi, lo, ab = orc.dd_entries(A, B, ta, 0, n, ii, jj)
    idx = torch.from_numpy(ii + jj * n).cuda()
    vals = Cdev[idx].cpu().numpy()
    return orc.errors(vals, hi, lo, ab)


def run_leg(eng, dA, dB, dC, n, steps, warmup, stream):
    import torch
    for _ in range(warmup):
        rc = eng.exec(dA, n, dB, n, dC, n)
        if rc:
            raise RuntimeError("exec failed: %d" % rc)
    torch.cuda.synchronize()
    eng.reset_stat()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the engine runs synchronously on the legacy default stream; events on it
    ev0.record(stream)
    for _ in range(steps):
        eng.exec(dA, n, dB, n, dC, n)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    s = eng.s
    return {"ms_per_step": ms, "gemm_ms": s.cannon_ms / max(s.n_exec, 1),
            "pack_ms": s.redist_ms / max(s.n_exec, 1), "reduce_ms": s.reduce_ms / max(s.n_exec, 1)}


def cpu_baseline(A, B, ta, n, budget_s=20.0):
    """The oracle's CPU restatement of the virtual-rank algorithm (BLAS local
    GEMMs, numpy) on a bounded sample: the k-slab 0 cuboids of the 4x2x3
    grid, i.e. one third of the 8000^3 work, repeated while under budget."""
    from oracle import oracle as orc
    cores = os.cpu_count()
    try:
        from threadpoolctl import threadpool_info
        cores = max([i.get("num_threads", 0) for i in threadpool_info()] + [1])
    except Exception:
        pass
    k0, kz = orc.block_spos_size(n, 3, 0)
    Ask = np.asfortranarray((A.T if ta else A)[:, k0:k0 + kz])
    Bsk = np.asfortranarray(B[k0:k0 + kz, :])
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
    if rank != 0:
        return
    n = args.size
    A, B = make_inputs(n, args.trans_a)
    steps, warm = max(args.steps, 1), max(args.warmup, 0)
    base = None
    for _ in range(warm):
        cpu_baseline(A, B, args.trans_a, n, budget_s=4.0)
    vals = []
    for _ in range(steps):
        base = cpu_baseline(A, B, args.trans_a, n, budget_s=4.0)
        vals.append(base["value"])
    v = float(np.median(vals))
    base["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "TFLOP/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": 2.0 * n * n * n / (v * 1e12) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "ca3dmm_exec M=N=K=%d transA=%d grid 4x2x3 (24 virtual ranks)"
                                   % (n, args.trans_a), "l2": "inputs larger than L2"},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "reference CPU path restated by the oracle (MPI + BLAS cannot be built here)"}
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
    """Configuration 4: one persistent grouped launch (captured in a CUDA graph)
    against one plain DMMA launch per GEMM."""
    import torch
    import ca3dmm_b200 as cb
    from oracle import oracle as orc
    torch.cuda.set_device(local)
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
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                fn()
            e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    # one plain DMMA launch (pack + GEMM) per product
    singles = [cb.GroupedGemm([m], [n], [k], [ta], [tb]) for m, n, k, ta, tb in probs]
    for i, g in enumerate(singles):
        g.set_stream(stream.cuda_stream, 0)

    def run_singles():
        for i, g in enumerate(singles):
            g.exec([dA[i]], [lda[i]], [dB[i]], [ldb[i]], [dC[i]], [ldc[i]])
    res["per_gemm_launches_ms"] = timed(run_singles, args.steps)
    for mode, sl, key in ((cb.GEMM_PLAIN, 0, "grouped_plain"), (cb.GEMM_OZAKI, 7, "grouped_ozaki7")):
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
    v = flops / (res["grouped_ozaki7_ms"] * 1e-3) / 1e12
    out = {"metric": METRIC, "value": v, "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": res["grouped_ozaki7_ms"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic",
           "config": {"workload": "%d independent GEMMs, m,n,k log-uniform in [64,4096], random "
                                  "trans, one grouped launch in a CUDA graph" % len(probs),
                      "total_flop": flops},
           "legs_ms": res,
           "legs_tflops": {k.replace("_ms", ""): flops / (t * 1e-3) / 1e12 for k, t in res.items()}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
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
    n = args.size
    A, B = make_inputs(n, args.trans_a)
    dA = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    dB = torch.from_numpy(B.ravel(order="F").copy()).cuda()
    dC = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.default_stream()
    flops = 2.0 * n * n * n

    legs = {}
    eng_plain = cb.Ca3dmmEngine(n, n, n, args.trans_a, 0, p=P)
    assert eng_plain.ok, "engine init failed"
    eng_plain.set_gemm_mode(cb.GEMM_PLAIN)
    eng_oz = None
    oz_slices = int(os.environ.get("CA3DMM_BENCH_SLICES", "7"))
    try:
        e = cb.Ca3dmmEngine(n, n, n, args.trans_a, 0, p=P)
        if e.ok and e.set_gemm_mode(cb.GEMM_OZAKI, oz_slices) == 0 and \
                e.exec(dA, n, dB, n, dC, n) == 0:
            eng_oz = e
    except Exception:
        eng_oz = None

    # plain leg
    legs["plain"] = run_leg(eng_plain, dA, dB, dC, n, 1, args.warmup, stream)
    legs["plain"]["err"] = error_vs_dd(dC, A, B, args.trans_a, n)
    if eng_oz is not None:
        legs["ozaki"] = run_leg(eng_oz, dA, dB, dC, n, 1, args.warmup, stream)
        legs["ozaki"]["err"] = error_vs_dd(dC, A, B, args.trans_a, n)
    head = "ozaki" if eng_oz is not None else "plain"
    eng = eng_oz if eng_oz is not None else eng_plain

    # timed region (headline leg), clocks sampled meanwhile
    sampler = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    res = run_leg(eng, dA, dB, dC, n, args.steps, 0, stream)
    clocks = sampler.stop()
    ms = res["ms_per_step"]
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = world * flops / (ms * 1e-3) / 1e12
    # also time the other leg over the same number of steps (reported beside)
    other = "plain" if head == "ozaki" else None
    if other:
        r2 = run_leg(eng_plain, dA, dB, dC, n, max(2, args.steps // 2), 1, stream)
        legs["plain"].update(r2)

    # e2e: the same exec through the C ABI with host buffers, copies timed
    hA = torch.from_numpy(A.ravel(order="F").copy()).pin_memory()
    hB = torch.from_numpy(B.ravel(order="F").copy()).pin_memory()
    hC = torch.empty(n * n, dtype=torch.float64).pin_memory()
    e2e_steps = max(2, min(args.steps, 5))
    for _ in range(1):
        dA.copy_(hA, non_blocking=True); dB.copy_(hB, non_blocking=True)
        eng.exec(dA, n, dB, n, dC, n); hC.copy_(dC)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(e2e_steps):
        dA.copy_(hA, non_blocking=True)
        dB.copy_(hB, non_blocking=True)
        eng.exec(dA, n, dB, n, dC, n)
        hC.copy_(dC, non_blocking=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = ev0.elapsed_time(ev1) / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())

    peaks = measured_peaks()
    traffic = ncu_traffic()
    gemm_ms = res["gemm_ms"]
    if head == "ozaki":
        s = eng.s.ozaki_slices
        ops = flops * s * (s + 1) / 2           # INT8 ops of the slice products
        peak = 2.0 * peaks.get("bf16_tflops", 1590.0)
        roof = {"bound": "tensor", "achieved": ops / (gemm_ms * 1e-3) / 1e12, "peak": peak,
                "unit": "TFLOP/s", "peak_source": "2 x measured dense bf16 (INT8 dense rate)",
                "traffic": traffic.get("ozaki_gemm")}
    else:
        sm_mhz = peaks.get("sm_max_mhz", 1965.0)
        peak = 148 * 128 * sm_mhz * 1e6 / 1e12
        roof = {"bound": "tensor", "achieved": flops / (gemm_ms * 1e-3) / 1e12, "peak": peak,
                "unit": "TFLOP/s",
                "peak_source": "nominal FP64 DMMA rate 148 SM x 128 flop/clk x max SM clock",
                "traffic": traffic.get("dgemm_dmma")}
    roof["frac"] = roof["achieved"] / roof["peak"]
    launches_per_step = 4 if head == "plain" else 5
    out = {
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "ca3dmm_exec M=N=K=%d transA=%d transB=0, 24 virtual ranks, grid "
                               "4x2x3 (cuboid 2000x4000x2667), entries sign*(1+u)*2^e, e in [-8,8]"
                               % (n, args.trans_a),
                   "gemm": head, "ozaki_slices": eng.s.ozaki_slices if head == "ozaki" else None,
                   "l2": "inputs larger than L2 (512 MB per operand), no flush"},
        "legs": legs, "roofline": roof, "clocks": clocks,
        "e2e": {"value": world * flops / (e2e_ms * 1e-3) / 1e12, "unit": "TFLOP/s",
                "h2d_bytes_per_step": 2 * n * n * 8, "d2h_bytes_per_step": n * n * 8},
        "gpu_launches": launches_per_step * args.steps,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(A, B, args.trans_a, n)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
