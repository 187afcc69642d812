#!/usr/bin/env python
"""Benchmark: time-to-k-triplets of randomized_svd on the 100,000 x 30,000
count-like workload, FP32 (mixed) GPU path against the plain-f64 GPU path.

    python bench.py --gpus N --steps K --warmup W [--impl reference] [--workload randomized|las2]

One JSON line on rank 0.  A step is one randomized_svd call (rank 50, 10
oversamples, 3 power iterations, QR normaliser, seed 7) on an all-columns
MaskedCSRMatrix, the form in which the crate can run it.  `value` is seconds
per solve with the matrix resident in HBM (CUDA events, max over ranks);
`e2e` is the same through the public API from pinned host buffers (matrix
upload and result download inside the timed region).  Several GPUs run
independent replicas (weak scaling).  `--impl reference` times the CPU
restatement of the crate's path (oracle/, all host threads) on a row sample
of the same workload and scales it to the full matrix.
"""
from __future__ import annotations

import argparse
import ctypes as C
import faulthandler
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "single-svdlib_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

# workload (randomized_svd on the count-like matrix)
M_ROWS, N_COLS = 100_000, 30_000
TARGET_RANK, OVERSAMPLES, POWER_ITERS, SEED = 50, 10, 3, 7
GEN_SEED = 2024
WORKLOAD = ("randomized_svd 100000x30000 count-like CSR (lambda_j~Gamma(0.5,2), row nnz~LogNormal(ln600,0.5), "
            "values log1p(Poisson(lambda_j)+1)), rank 50 + 10 oversamples, 3 power iterations, QR, seed 7, "
            "MaskedCSRMatrix all columns")


# ------------------------------------------------------------------ data --
def generate(m=M_ROWS, n=N_COLS, seed=GEN_SEED):
    """Seeded synthetic count-like CSR.  Columns are drawn proportional to
    lambda_j with replacement and merged per row (realised nnz is reported)."""
    rng = np.random.default_rng(seed)
    lam = rng.gamma(0.5, 2.0, n)
    k = np.clip(np.rint(rng.lognormal(np.log(600.0), 0.5, m)), 1, n).astype(np.int64)
    cdf = np.cumsum(lam / lam.sum())
    cdf[-1] = 1.0
    rows = np.repeat(np.arange(m, dtype=np.int64), k)
    cols = np.searchsorted(cdf, rng.random(rows.size), side="right").astype(np.int64)
    np.minimum(cols, n - 1, out=cols)
    keys = rows * n + cols
    keys.sort()
    keep = np.ones(keys.size, dtype=bool)
    keep[1:] = keys[1:] != keys[:-1]
    rows, cols = np.divmod(keys[keep], n)
    del keys, keep
    indptr = np.zeros(m + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=m), out=indptr[1:])
    vals = np.log1p(rng.poisson(lam[cols]) + 1.0)
    return indptr, cols, vals


def stage(msg):
    """Progress marker on stderr (flushed), so a crash can be located."""
    print(f"[bench] {time.strftime('%H:%M:%S')} {msg}", file=sys.stderr, flush=True)


def load_or_generate(rank, world):
    path = os.path.join(tempfile.gettempdir(), f"svdb_bench_{M_ROWS}x{N_COLS}_{GEN_SEED}.npz")
    if rank == 0 and not os.path.exists(path):
        indptr, cols, vals = generate(M_ROWS, N_COLS, GEN_SEED)
        tmp = path + f".{os.getpid()}.npz"
        np.savez(tmp, indptr=indptr, cols=cols, vals=vals)
        os.replace(tmp, path)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    d = np.load(path)
    return d["indptr"], d["cols"], d["vals"]


# ---------------------------------------------------------------- clocks --
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.out:
            return None
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return None
        def num(x):
            try:
                return float(x)
            except ValueError:
                return float("nan")
        sm = [num(r[1]) for r in rows]
        mx = max(num(r[2]) for r in rows)
        loaded = [s for s, r in zip(sm, rows) if num(r[3]) > 200] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------- helpers --
def peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(name):
    """Bytes per launch from a committed ncu summary line 'traffic_bytes_per_launch: <n>'."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_reference(indptr, cols, vals, threads, sample_rows, omega):
    """The CPU restatement of randomized_svd (oracle/) on the first `sample_rows` rows.

    Returns (estimated seconds for the full matrix, measured seconds, sample nnz): the
    sparse-product time is scaled by the nnz ratio, the m-row dense work (QR of Y,
    U = Q U_B) by the row ratio, and the n-row / small-SVD work is taken as measured."""
    import oracle as O
    O.set_threads(threads)
    nnz_s = int(indptr[sample_rows])
    A = {"nrows": sample_rows, "ncols": N_COLS, "indptr": indptr[: sample_rows + 1], "indices": cols[:nnz_s],
         "data": vals[:nnz_s]}
    t0 = time.perf_counter()
    r = O.randomized(A, TARGET_RANK, OVERSAMPLES, POWER_ITERS, "QR", omega=omega)
    measured = time.perf_counter() - t0
    t = r["times"]
    full = t["sparse"] * (len(vals) / nnz_s) + t["rows"] * (M_ROWS / sample_rows) + t["fixed"]
    return full, measured, nnz_s


# ------------------------------------------------------------------- main --
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-sample-rows", type=int, default=20000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=float, default=1.0, help="shrink both dimensions (smoke runs only)")
    args = ap.parse_args()
    faulthandler.enable()
    global M_ROWS, N_COLS
    if args.scale != 1.0:
        M_ROWS, N_COLS = int(M_ROWS * args.scale), int(N_COLS * args.scale)
        args.cpu_sample_rows = min(args.cpu_sample_rows, M_ROWS)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)

    if args.impl == "reference":
        if rank != 0:
            return 0
        indptr, cols, vals = load_or_generate(0, 1)
        nnz = len(vals)
        om = np.random.default_rng(SEED).standard_normal((N_COLS, TARGET_RANK + OVERSAMPLES))
        for _ in range(args.warmup):
            cpu_reference(indptr, cols, vals, threads, min(1000, args.cpu_sample_rows), om)
        times = []
        for _ in range(args.steps):
            t, measured, nnz_s = cpu_reference(indptr, cols, vals, threads, args.cpu_sample_rows, om)
            times.append(t)
        v = statistics.mean(times)
        sample = (f"first {args.cpu_sample_rows} of {M_ROWS} rows ({nnz_s} of {nnz} nnz), full randomized_svd on "
                  f"the CPU restatement ({measured:.1f} s measured); sparse-product time scaled by nnz, m-row "
                  f"dense work by rows")
        print(json.dumps({
            "impl": "reference", "metric": "time-to-k-triplets (s), randomized_svd k=50", "value": v, "unit": "s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "nnz": nnz},
            "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
        return 0

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))

    from single_svdlib import CsrMatrix, MaskedCSRMatrix, _abi
    from single_svdlib._core import check, options, rec_from_c
    L = _abi.lib()

    stage("load matrix")
    indptr, cols, vals = load_or_generate(rank, world)
    m, n, nnz = M_ROWS, N_COLS, len(vals)
    # pinned host copies: the e2e inputs
    h_indptr = torch.from_numpy(indptr.astype(np.uint64).view(np.int64)).pin_memory()
    h_cols = torch.from_numpy(cols.astype(np.uint64).view(np.int64)).pin_memory()
    h_vals = torch.from_numpy(vals).pin_memory()

    def create(pinned=True):
        h = C.c_void_p()
        check(L.svdb_matrix_create_csr(m, n, nnz, h_indptr.data_ptr(), h_cols.data_ptr(), h_vals.data_ptr(),
                                       C.byref(h)))
        mask = np.ones(n, np.uint8)
        hm = C.c_void_p()
        check(L.svdb_masked_new(h, mask.ctypes.data, n, C.byref(hm)))
        return h, hm

    stage("upload")
    parent, masked = create()
    stream = torch.cuda.Stream()

    def solve(handle, precision, on_device, s=None):
        o = options(precision=precision, result_on_device=on_device)
        o.stream = s.cuda_stream if s is not None else None
        r = _abi.svdb_rec()
        check(L.svdb_randomized_svd(handle, TARGET_RANK, OVERSAMPLES, POWER_ITERS, 0, 0, 1, SEED, 0, C.byref(o),
                                    C.byref(r)))
        return r

    def timed(fn, k):
        recs = []
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            recs.append(fn())
        e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        return e0.elapsed_time(e1) / k, recs

    # ---- mixed (headline) and plain f64, inputs resident in HBM
    stage("warmup")
    for _ in range(args.warmup):
        L.svdb_rec_free(C.byref(solve(masked, "mixed", 1, stream)))
        L.svdb_rec_free(C.byref(solve(masked, "f64", 1, stream)))
    launches0 = L.svdb_kernel_launches()
    with ClockSampler(local) as clk:
        ms_mixed, recs = timed(lambda: solve(masked, "mixed", 1, stream), args.steps)
    launches = L.svdb_kernel_launches() - launches0
    clocks = clk.summary()
    for r in recs:
        L.svdb_rec_free(C.byref(r))
    stage("f64 timing")
    ms_f64, recs = timed(lambda: solve(masked, "f64", 1, stream), max(2, args.steps // 2))
    for r in recs:
        L.svdb_rec_free(C.byref(r))
    # sigma error of the FP32 path against the f64 path (same seed, so the same Omega); untimed
    sig = {}
    for prec in ("mixed", "f64"):
        r = solve(masked, prec, 0)
        sig[prec] = rec_from_c(r).s
        L.svdb_rec_free(C.byref(r))
    sigma_err = float(np.max(np.abs(sig["mixed"] - sig["f64"]) / np.abs(sig["f64"])))

    # ---- e2e: upload from pinned host memory + solve + host results, every step
    stage("e2e")

    def e2e_step():
        h, hm = create()
        r = solve(hm, "mixed", 0)
        L.svdb_rec_free(C.byref(r))
        L.svdb_matrix_destroy(hm)
        L.svdb_matrix_destroy(h)
        return None

    e2e_step()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if world > 1:
        torch.distributed.barrier()
    h2d = 8 * (m + 1) + 8 * nnz + 8 * nnz
    d2h = 8 * (m * TARGET_RANK + TARGET_RANK + TARGET_RANK * n)

    # ---- roofline of the dominant kernel: FP32 SpMM (A Z and A^T Y, l = 60)
    l = TARGET_RANK + OVERSAMPLES
    Xn = torch.randn(n, l, device="cuda", dtype=torch.float32)
    Ym = torch.randn(m, l, device="cuda", dtype=torch.float32)
    Yo = torch.empty(m, l, device="cuda", dtype=torch.float32)
    Zo = torch.empty(n, l, device="cuda", dtype=torch.float32)
    reps = 20

    def spmm_ms(transpose):
        x, y = (Ym, Zo) if transpose else (Xn, Yo)
        for _ in range(3):
            check(L.svdb_multiply_with_dense_device(masked, x.data_ptr(), l, y.data_ptr(), int(transpose), 1,
                                                    stream.cuda_stream))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            check(L.svdb_multiply_with_dense_device(masked, x.data_ptr(), l, y.data_ptr(), int(transpose), 1,
                                                    stream.cuda_stream))
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    stage("spmm roofline")
    ms_ax, ms_atx = spmm_ms(False), spmm_ms(True)
    bytes_ax = nnz * 8 + (m + 1) * 8 + n * l * 4 + m * l * 4
    bytes_atx = nnz * 8 + (n + 1) * 8 + m * l * 4 + n * l * 4
    gbs_ax, gbs_atx = bytes_ax / ms_ax / 1e6, bytes_atx / ms_atx / 1e6
    peak, peak_kind = peak_hbm()
    dominant = "spmm_csc_AtY" if ms_atx >= ms_ax else "spmm_csr_AZ"
    ach = gbs_atx if ms_atx >= ms_ax else gbs_ax

    ms_mixed = max_over_ranks(ms_mixed, world)
    ms_f64 = max_over_ranks(ms_f64, world)
    e2e_s = max_over_ranks(e2e_s, world)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        stage("cpu baseline")
        om = np.random.default_rng(SEED).standard_normal((n, l))
        t, measured, nnz_s = cpu_reference(indptr, cols, vals, threads, args.cpu_sample_rows, om)
        cpu = {"value": t, "unit": "s", "cores": threads, "kind": "port",
               "sample": f"first {args.cpu_sample_rows} of {m} rows ({nnz_s} of {nnz} nnz), full randomized_svd "
                         f"on the CPU restatement ({measured:.1f} s measured); sparse-product time scaled by nnz, "
                         f"m-row dense work by rows"}

    if rank == 0:
        line = {
            "metric": "time-to-k-triplets (s), randomized_svd k=50, FP32 GPU (sigma rel err vs f64 stated)",
            "value": ms_mixed / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_mixed, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nrows": m, "ncols": n, "nnz": nnz, "target_rank": TARGET_RANK,
                       "n_oversamples": OVERSAMPLES, "n_power_iters": POWER_ITERS, "normalizer": "QR",
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (FP32 CSR + CSC ~ %.0f MB)" % (nnz * 16 / 1e6)},
            "f64_value": ms_f64 / 1e3, "mixed_speedup_vs_f64": ms_f64 / ms_mixed,
            "sigma_rel_err_vs_f64": sigma_err,
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "traffic": profiled_traffic("spmm_randomized_100kx30k.md"), "kernel": dominant,
                         "peak_source": peak_kind,
                         "spmm_csr_AZ": {"ms": ms_ax, "gbs": gbs_ax, "bytes": bytes_ax},
                         "spmm_csc_AtY": {"ms": ms_atx, "gbs": gbs_atx, "bytes": bytes_atx}},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    stage("teardown")
    L.svdb_matrix_destroy(masked)
    L.svdb_matrix_destroy(parent)
    if world > 1:
        torch.distributed.destroy_process_group()
    stage("done")
    return 0


if __name__ == "__main__":
    sys.exit(main())
