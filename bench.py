"""Benchmark: backward-Euler 128^3 step (FP32 PCG + FP64 refinement to a 1e-8
relative residual) and CSR SpMV HBM throughput at 256^3.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl piro|reference]

One JSON line on rank 0.  A "step" is one backward-Euler time step of the
128^3 variable-alpha heat problem (seeded synthetic inputs; the trajectory of
20 steps repeats).  `value` is device time per step with inputs resident in
HBM; `e2e` is the same through host buffers (pinned H2D of u_n, D2H of
u_{n+1} inside the timed region).  Under torchrun every rank runs its own
replica (one process per GPU, barrier + max over ranks).
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

METRIC = "BE 128³ step ms at 1e-8 FP64 residual, learned-PCG vs plain; SpMV HBM GB/s"
L2_BYTES = 126 * 2 ** 20


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_metrics(kernel):
    """The figures of `kernel`'s committed ncu summary (profiles/<kernel>_128.md):
    `traffic_bytes_per_launch: N` and every `metric [unit] = value` line, as
    {name: float}.  Empty when the summary is absent."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_128.md")
    out = {}
    try:
        with open(path) as f:
            for line in f:
                line = line.strip()
                if line.startswith("traffic_bytes_per_launch:"):
                    out["traffic_bytes_per_launch"] = float(line.split(":")[1])
                elif " = " in line and "[" in line:
                    name, val = line.split(" = ", 1)
                    try:
                        out[name.split(" [")[0].strip()] = float(val.replace(",", ""))
                    except ValueError:
                        pass
    except OSError:
        pass
    return out


def load_tflops_peak():
    """Dense BF16 TFLOP/s (burst: the network applies are short kernels)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["bf16_tflops"])
    return 1590.0


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, period_ms: int = 50):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(gpu_index), "-lms", str(period_ms)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [ln.strip().split(", ") for ln in self.f.read().splitlines() if ln.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ problem
WORKLOAD = ("heat backward Euler 128^3, smoothed log-normal alpha (sigma 1.5, filter 8, seed 2), "
            "dt = 50x explicit limit, Jacobi-PCG to a 1e-8 FP64 relative residual")


def bench_config(cfg, world):
    """The `config` both arms print (identical, so the two lines describe the
    same problem): the workload, its grid and the nonzeros of A = I - dt
    diag(alpha) L (the Laplacian's pattern: 7N - 2(nx ny + ny nz + nx nz))."""
    nx, ny, nz = cfg["n"]
    N = nx * ny * nz
    return {"workload": WORKLOAD, "grid": [nx, ny, nz], "nnz_A": 7 * N - 2 * (nx * ny + ny * nz + nx * nz),
            "steps_in_trajectory": cfg["steps"], "parallelism": f"replicas x{world}"}


def be_problem(torch, ops, cfg):
    nx, ny, nz = cfg["n"]
    N = nx * ny * nz
    alpha = torch.from_numpy(cfg["alpha"]).cuda()
    L = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    ops.csr_rowscale(L[0], L[2], alpha)
    I = ops.csr_identity(N)
    A = ops.csrgeam2(N, I, -float(cfg["dt"]), L)
    del L, I
    return A, alpha


def spmv_section(torch, ops, steps, warmup, peak):
    """CSR / COO / HT / matrix-free 7-point forward-Euler steps at 256^3."""
    from piro_b200 import workloads as W
    cfg = W.spmv_256()
    nx, ny, nz = cfg["n"]
    N = nx * ny * nz
    u = torch.from_numpy(cfg["u"]).cuda()
    alpha = torch.from_numpy(cfg["alpha"]).cuda()
    out = torch.empty_like(u)
    dt = 0.01
    res = {}

    def timeit(fn, n_iter):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n_iter):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n_iter

    A = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    ops.csr_rowscale(A[0], A[2], alpha)
    nnz = A[2].numel()
    ms = timeit(lambda: ops.csr_fe_step(nx, ny, nz, A, dt, u, out), steps)
    byt = 8 * nnz + 4 * (N + 1) + 4 * N + 4 * N
    res["csr"] = {"ms": ms, "gbs": byt / ms / 1e6, "frac": byt / ms / 1e6 / peak, "bytes": byt, "nnz": nnz}
    ms = timeit(lambda: ops.stencil_fe_step(nx, ny, nz, dt, u, out, alpha=alpha), steps)
    byt = 12 * N
    res["stencil"] = {"ms": ms, "gbs": byt / ms / 1e6, "frac": byt / ms / 1e6 / peak, "bytes": byt}
    ts = ops.ht_table_size(nnz, N, 1)
    keys, vals = ops.ht_build(N, *A, ts)
    # the table streams through once (8-byte key + 4-byte value per slot), u
    # read, out written, the row order read
    byt = 12 * ts + 12 * N
    order = ops.ht_row_order(N, ts)
    stage = ops.ht_stage(N)
    ms = timeit(lambda: ops.ht_spmv_staged(nx, ny, nz, keys, vals, dt, order, stage, u, out, fe=True), steps)
    res["ht"] = {"ms": ms, "gbs": byt / ms / 1e6, "frac": byt / ms / 1e6 / peak, "bytes": byt, "slots": ts,
                 "rows": "table read with the rows in home-slot order (piro_ht_row_order, once per table), "
                         "each row's values staged in a 32-byte record, then applied in row order",
                 "stage_bytes": 32 * N,
                 "bytes_definition": "12 ts (keys and values, every slot) + 12 N (u, out, row order); the "
                                     "stage's 64 N bytes (written, read back) are not counted"}
    del stage
    ms = timeit(lambda: ops.ht_spmv_ordered(nx, ny, nz, keys, vals, dt, order, u, out, fe=True), steps)
    res["ht_one_pass"] = {"ms": ms, "gbs": byt / ms / 1e6, "frac": byt / ms / 1e6 / peak}
    ms = timeit(lambda: ops.ht_spmv(nx, ny, nz, keys, vals, dt, u, out, fe=True), max(3, steps // 4))
    res["ht_row_major"] = {"ms": ms, "gbs": byt / ms / 1e6, "frac": byt / ms / 1e6 / peak}
    del order
    del keys, vals
    rows = torch.repeat_interleave(torch.arange(N, device="cuda", dtype=torch.int32),
                                   (A[0][1:] - A[0][:-1]).to(torch.int64))
    coo = (rows, A[1], A[2])
    rowstart = ops.coo_row_index(N, rows)
    ms = timeit(lambda: ops.coo_step_indexed(N, rowstart, A[1], A[2], dt, u, out, fe=True), steps)
    byt = 8 * nnz + 4 * (N + 1) + 8 * N  # cols, vals, the row index, u, out
    res["coo"] = {"ms": ms, "gbs": byt / ms / 1e6, "frac": byt / ms / 1e6 / peak, "bytes": byt,
                  "rows": "row index built once per operator (piro_coo_row_index)"}
    ms = timeit(lambda: ops.coo_spmv(N, coo, dt, u, out, fe=True), steps)
    byt = 12 * nnz + 8 * N
    res["coo_segsum"] = {"ms": ms, "gbs": byt / ms / 1e6, "frac": byt / ms / 1e6 / peak, "bytes": byt}
    del rowstart
    del A, coo, rows
    torch.cuda.empty_cache()
    res["cpu_baseline"] = spmv_cpu_baseline(peak)
    return res


def spmv_cpu_baseline(peak):
    """PIRO's own SpMV kernels (SpMVCSR.cl, SpMVCOO.cl, SpMVHT.cl compiled
    for the host by oracle/Makefile, the NDRange run as an OpenMP loop): CSR
    at 256^3 on all host threads and on one; COO and HT at 32^3 only, since
    as written they cost O(N nnz) and O(N^2) per step.  None when the
    reference build is absent."""
    from oracle import oracle as O
    from piro_b200 import workloads as W
    try:
        R = O.Ref()
    except (FileNotFoundError, OSError):
        return None
    out = {"kind": "reference", "source": "PIRO's .cl kernels compiled for the host (oracle/_ref)"}
    cfg = W.spmv_256()
    nx, ny, nz = cfg["n"]
    N = nx * ny * nz
    L = O.laplacian(nx, ny, nz, 3, np.float32(1.0))
    A = (L[0], L[1], O.csr_rowscale(N, L[0], L[2], cfg["alpha"]))
    nnz = len(A[2])
    byt = 8 * nnz + 4 * (N + 1) + 8 * N
    nthr = O.num_threads()
    for th, reps in ((nthr, 3), (1, 1)):
        O.set_threads(th)
        R.spmv_par("csr", nx, ny, nz, A, 0.01, cfg["u"])
        t0 = time.perf_counter()
        for _ in range(reps):
            R.spmv_par("csr", nx, ny, nz, A, 0.01, cfg["u"])
        ms = (time.perf_counter() - t0) * 1e3 / reps
        out[f"csr_256_{'all' if th == nthr else 'one'}_threads"] = {
            "ms": round(ms, 2), "cores": th, "gbs": round(byt / ms / 1e6, 1), "bytes": byt,
            "sample": f"SpMVCSR.cl at 256^3 ({N} rows, {nnz} nonzeros), mean of {reps}"}
    O.set_threads(nthr)
    del A, L
    n = 32
    N = n ** 3
    u = np.random.default_rng(1).random(N).astype(np.float32)
    L = O.laplacian(n, n, n, 3, np.float32(1.0))
    rows = np.repeat(np.arange(N, dtype=np.int32), np.diff(L[0]))
    t0 = time.perf_counter()
    R.spmv_par("coo", n, n, n, (rows, L[1], L[2]), 0.01, u)
    ms = (time.perf_counter() - t0) * 1e3
    out["coo_32_all_threads"] = {"ms": round(ms, 1), "cores": nthr,
                                 "sample": f"SpMVCOO.cl at 32^3 ({N} rows, {len(L[2])} nonzeros; every row scans all "
                                           "nonzeros), one step"}
    ts = O.ht_table_size_build(len(L[2]))
    keys, vals = O.ht_build(N, *L, ts)
    t0 = time.perf_counter()
    R.spmv_par("ht", n, n, n, (keys.astype(np.int32), vals), 0.01, u)
    ms = (time.perf_counter() - t0) * 1e3
    out["ht_32_all_threads"] = {"ms": round(ms, 1), "cores": nthr,
                                "sample": f"SpMVHT.cl at 32^3 ({N} rows, {ts}-slot table; every row looks up all N "
                                          "columns), one step"}
    return out


def config_sections(torch, peak):
    """Configuration 1 (32^3 forward-Euler heat, 100 steps) and the advection
    part of configuration 2 (256^3 upwind, csrgeam-merged operator, 1000
    steps), each replayed from a CUDA graph of two steps."""
    from piro_b200 import fe
    from piro_b200 import workloads as W
    out = {}
    c = W.heat_fe_32()
    nx, ny, nz = c["n"]
    N = nx * ny * nz
    run = fe.FeRunner(nx, ny, nz, torch.from_numpy(c["alpha"]).cuda(), float(c["dt"]))
    u0 = torch.from_numpy(c["u0"]).cuda()
    replay = run.capture(u0)
    replay(5)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    replay(c["steps"] // 2)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out["heat_fe_32"] = {"steps": c["steps"], "ms_total": round(ms, 4), "us_per_step": round(1e3 * ms / c["steps"], 2),
                         "note": "graph replays of two steps each, one fused kernel per step (zero-filled result, "
                                 "SpMVCSR-order update, setBC), captured once; 32^3 = 2.3 MB per step is "
                                 "launch-bound and L2-resident by size (no flush between the graph's steps)"}
    c = W.advection(256)
    nx, ny, nz = c["n"]
    N = nx * ny * nz
    run = fe.AdvectionRunner(nx, ny, nz, torch.from_numpy(c["v"]).cuda(), float(c["dt"]), float(c["gnorm"]))
    nnz = run.A[2].numel()
    u0 = torch.from_numpy(c["u0"]).cuda()
    replay = run.capture(u0)
    replay(2)
    steps = c["steps"]
    torch.cuda.synchronize()
    e0.record()
    replay(steps // 2)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    byt = 8 * nnz + 4 * (N + 1) + 8 * N
    out["advection_256"] = {"steps": steps, "ms_per_step": round(ms, 4), "nnz": nnz, "gbs": round(byt / ms / 1e6, 1),
                            "frac": round(byt / ms / 1e6 / peak, 4),
                            "note": "per step: one fused kernel (zero-filled result, SpMVCSR-order update, setBC)"}
    del run
    torch.cuda.empty_cache()
    return out


def assembly_section(torch, ops, peak):
    """Assembly of the CSR Laplacian (central): on the device at 32^3 and
    256^3, and PIRO's own host assembly (CSR::stencils::laplacian_cd, with
    its std::find over the whole column array per boundary row) at 32^3,
    the largest size where it is tractable (it is O(nnz * boundary rows))."""
    out = {}
    for n in (32, 256):
        N = n ** 3
        for _ in range(2):
            A = ops.csr_laplacian(n, n, n, 3, 1.0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            A = ops.csr_laplacian(n, n, n, 3, 1.0)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 5
        nnz = A[2].numel()
        byt = 4 * (N + 1) + 8 * nnz
        out[f"csr_laplacian_{n}"] = {"ms": round(ms, 4), "nnz": nnz, "bytes_written": byt,
                                     "gbs": round(byt / ms / 1e6, 1), "frac": round(byt / ms / 1e6 / peak, 4)}
        del A
    # v . grad merge (operator&, csrgeam count + scan + fill) at 256^3 of the
    # upwind gradients; bytes: sum 8 nnz_in + 12 N (v) + 8 nnz_out + 4 (N+1)
    n = 256
    N = n ** 3
    G = [ops.csr_gradient(n, n, n, 1, a, 2.0) for a in range(3)]
    v = torch.rand(3 * N, device="cuda")
    for _ in range(2):
        D = ops.csrgeam3(N, *G, v)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        D = ops.csrgeam3(N, *G, v)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 5
    nnz_in = sum(int(g[2].numel()) for g in G)
    byt = 8 * nnz_in + 12 * N + 8 * int(D[2].numel()) + 4 * (N + 1)
    out["csrgeam3_256"] = {"ms": round(ms, 4), "nnz_out": int(D[2].numel()), "bytes": byt,
                           "gbs": round(byt / ms / 1e6, 1), "frac": round(byt / ms / 1e6 / peak, 4),
                           "note": "count, one device scan, fill (the reference: N scan launches)"}
    del G, D, v
    torch.cuda.empty_cache()
    try:  # PIRO's own host code (oracle/_ref), when it was built
        from oracle import oracle as O
        R = O.Ref()
        t0 = time.perf_counter()
        R.laplacian(32, 32, 32, 3, np.float32(1.0))
        out["reference_host_32_ms"] = round((time.perf_counter() - t0) * 1e3, 1)
    except (FileNotFoundError, OSError):
        out["reference_host_32_ms"] = None
    return out


def next_rows_section(torch, ops, peak):
    """DENSE forward Euler at 34^3 (N = 39,304: a 6.2 GB matrix, HBM stream)
    and scheme 27: the banded LU (factor once, solve per step) at 34^3, and
    PIRO's own factorization on the Test/LUDecomp.ini shape (5^3 with ghosts,
    central, l = 5) on the device and by the reference's code on the host."""
    out = {}
    n = 34
    N = n ** 3
    A = ops.dense_laplacian(n, n, n, 3, 1.0)
    u = torch.rand(N, device="cuda")
    x = torch.empty_like(u)
    for _ in range(3):
        ops.dense_fe_step(A, 0.01, u, x)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(10):
        ops.dense_fe_step(A, 0.01, u, x)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 10
    byt = 4 * N * N + 8 * N
    out["dense_fe_34"] = {"kernel": "k_dense_fe_bulk", "N": N, "ms": round(ms, 4), "bytes": byt,
                          "gbs": round(byt / ms / 1e6, 1), "frac": round(byt / ms / 1e6 / peak, 4),
                          "note": "A (4 N^2 bytes) read once per step, larger than L2"}
    del A
    torch.cuda.empty_cache()

    L = ops.csr_laplacian(n, n, n, 3, 1.0)
    ts = ops.ht_table_size(L[2].numel(), N, 1)
    keys, vals = ops.ht_build(N, *L, ts)
    lu = ops.HtLu(N, n * n, keys, vals, ts, 1.0, -0.05)  # untimed: the first call allocates the band
    del lu
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    lu = ops.HtLu(N, n * n, keys, vals, ts, 1.0, -0.05)
    e1.record()
    torch.cuda.synchronize()
    f_ms = e0.elapsed_time(e1)
    b = torch.rand(N, device="cuda")
    lu.solve(b, x)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        lu.solve(b, x)
    e1.record()
    torch.cuda.synchronize()
    s_ms = e0.elapsed_time(e1) / 5
    out["scheme27_band_34"] = {"N": N, "bandwidth": n * n, "band_bytes": lu.nbytes, "factor_ms": round(f_ms, 2),
                               "solve_ms": round(s_ms, 3), "matrix": "I - 0.05 L (central, h = 1)",
                               "method": "FP64 banded LU with partial pivoting by 16-column panels (the panel in "
                                         "shared memory, then the exchanges and U rows right of it, then a tiled "
                                         "update below), FP64 solve in one block"}
    del lu, keys, vals, L
    torch.cuda.empty_cache()

    # PIRO's factorization, LUDecomp.ini shape: n = 3 3 3 (+2), l = 5, reference table size
    nx = 5
    Nl = nx ** 3
    norm = float(np.float32(float(np.float32(5.0) / np.float32(nx - 2)) ** 2))  # operatorlaplacian.cpp:33
    L = ops.csr_laplacian(nx, nx, nx, 3, norm)
    ts = ops.ht_table_size(L[2].numel(), Nl, 0)
    keys, vals = ops.ht_build(Nl, *L, ts)
    k0, v0 = keys.clone(), vals.clone()
    ops.ht_lu_reference(Nl, keys, vals, ts)
    reps = 5
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        keys.copy_(k0)
        vals.copy_(v0)
        ops.ht_lu_reference(Nl, keys, vals, ts)
    torch.cuda.synchronize()
    g_ms = (time.perf_counter() - t0) * 1e3 / reps
    ref_ms = None
    try:  # CPU baseline of this row: PIRO's own code (oracle/_ref), when it was built
        from oracle import oracle as O
        R = O.Ref()
        kh = k0.cpu().numpy().astype(np.int32)
        vh = v0.cpu().numpy()
        t0 = time.perf_counter()
        for _ in range(reps):
            k, v = kh.copy(), vh.copy()
            R.ht_lu(Nl, k, v, ts)
        ref_ms = (time.perf_counter() - t0) * 1e3 / reps
        same = bool(np.array_equal(k.astype(np.int64), keys.cpu().numpy()))
    except (FileNotFoundError, OSError):
        same = None
    out["scheme27_reference_5"] = {"N": Nl, "table_slots": ts, "device_ms": round(g_ms, 3),
                                   "reference_host_ms": None if ref_ms is None else round(ref_ms, 3),
                                   "same_table": same,
                                   "note": "reference: PIRO's fill-in and lu_decompHT.cl compiled for the host, "
                                           "without its per-round full-table transfers"}
    return out


def learned_section(torch, ops, cfg, A, alpha, plain_ms, plain_iters, steps, tflops_peak, l2_flush):
    """Configuration 4: the backward-Euler step with the learned preconditioner
    (the network trained on the device on seeds 100-199 by
    `python -m piro_b200.learned`, weights in piro_b200/data) inside flexible
    CG, against plain Jacobi-PCG on the same step; plus the held-out fields
    (seeds 200-209) solved both ways."""
    from piro_b200 import learned as LP
    nx, ny, nz = cfg["n"]
    N = nx * ny * nz
    w = np.load(os.path.join(ROOT, "piro_b200", "data", "pcnet_be128.npy"))
    net = ops.PCNet(seed=0)
    net.set_params(w)
    sv = ops.BESolver(nx, ny, nz, A, alpha, stencil=(float(cfg["dt"]), 1.0))
    sv.set_preconditioner(net)
    u0 = torch.from_numpy(cfg["u0"]).cuda()
    u, x = u0.clone(), torch.empty_like(u0)
    for _ in range(2):
        sv.solve(u, x, rtol=1e-8)
    sv.pc_stats(reset=True)
    sv.kernel_stats(reset=True)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    iters, fb, worst = [], 0, 0.0
    u.copy_(u0)
    for i in range(steps):
        if i % cfg["steps"] == 0:
            u.copy_(u0)
        l2_flush()  # as for the plain step
        ev[i][0].record()
        info = sv.solve(u, x, rtol=1e-8)
        ev[i][1].record()
        u, x = x, u
        iters.append(info.inner_iterations)
        fb += info.fallbacks
        worst = max(worst, info.rel_residual)
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev) / steps
    napply, apply_ms = sv.pc_stats(reset=True)
    _, _, launches = sv.kernel_stats(reset=True)
    sv.close()
    n_int = (nx - 2) * (ny - 2) * (nz - 2)
    alg_flops = 2 * 27 * (2 * 16 + 16 * 16 + 16 * 16 + 16 * 1) * n_int  # the network's multiply-adds
    avg_apply = apply_ms / max(1, napply)
    held_seeds = list(range(200, 210))
    LP.prefetch_alpha(nx, held_seeds)
    held = LP.compare(torch, ops, net, nx, held_seeds)
    net.close()
    return {
        "ms_per_step": round(ms, 4), "inner_iterations_mean": float(np.mean(iters)), "fallbacks": fb,
        "worst_rel_residual": worst, "plain_ms_per_step": plain_ms, "plain_iterations_mean": plain_iters,
        "speedup_vs_plain": round(plain_ms / ms, 4), "iteration_ratio": round(plain_iters / float(np.mean(iters)), 3),
        "network_applies_per_step": napply / steps, "apply_ms": round(avg_apply, 4),
        "apply_tflops": round(alg_flops / avg_apply / 1e9, 1),
        "apply_frac_of_bf16_peak": round(alg_flops / avg_apply / 1e9 / tflops_peak, 4),
        "kernel_launches_per_step": launches / steps,
        "held_out": dict(LP.summary(held), seeds=[held_seeds[0], held_seeds[-1]]),
        "note": "network applies on the tensor cores (tcgen05, 4 layers); the network preconditions the first "
                "flexible-CG iteration of each refinement sweep, Jacobi the rest (in one persistent launch); "
                "plain = Jacobi-PCG in the persistent single-launch solver",
    }


def training_section(torch, ops, tflops_peak, steps=30, batch=16, crop=32):
    """Training throughput of the learned preconditioner's network: one step =
    forward, masked-MSE loss, backward and Adam on `batch` crops of crop^3
    interior cells (+ a ghost layer), the batch the training recipe uses
    (piro_b200/learned.py: 10 000 pairs of 32^3 crops, batches of 16).  Both
    engines: every convolution on tcgen05 (forward, data and weight
    gradients), and the CUDA-core kernels.  Inputs are seeded random crops
    (the kernels' cost does not depend on the values)."""
    m = crop + 2
    N = m ** 3
    rng = np.random.default_rng(5)
    r = torch.from_numpy(rng.standard_normal(batch * N).astype(np.float32)).cuda()
    f = torch.from_numpy((0.5 * rng.standard_normal(batch * N)).astype(np.float32)).cuda()
    t = torch.from_numpy((0.1 * rng.standard_normal(batch * N)).astype(np.float32)).cuda()
    mk = torch.from_numpy((rng.random(batch * N) > 0.3).astype(np.float32)).cuda()
    n_int = batch * crop ** 3
    # multiply-adds of one step: forward 30 240 N, data gradients of layers 2-4
    # (16x16, 16x16, 1x16 per tap) and weight gradients of all four layers
    fwd = 2 * 27 * (2 * 16 + 16 * 16 + 16 * 16 + 16) * n_int
    bwd_data = 2 * 27 * (16 * 16 + 16 * 16 + 16) * n_int
    bwd_w = fwd
    flops = fwd + bwd_data + bwd_w
    out = {"batch": batch, "crop": crop, "cells_per_step": batch * N, "flop_per_step": flops}
    for name, tc in (("tensor_cores", True), ("cuda_cores", False)):
        net = ops.PCNet(seed=0)
        net.set_engine(tc)
        for _ in range(3):
            net.loss_grad(m, m, m, r, f, t, mk, batch=batch, want_loss=False)
            net.adam_step(1e-4)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            net.loss_grad(m, m, m, r, f, t, mk, batch=batch, want_loss=False)
            net.adam_step(1e-4)
        e1.record()
        loss, _ = net.loss_grad(m, m, m, r, f, t, mk, batch=batch)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[name] = {"ms_per_step": round(ms, 3), "pairs_per_s": round(batch / ms * 1e3, 1),
                     "tflops": round(flops / ms / 1e9, 1), "frac_of_bf16_peak": round(flops / ms / 1e9 / tflops_peak, 4),
                     "loss_finite": bool(np.isfinite(loss))}
        net.close()
    out["speedup_tensor_vs_cuda_cores"] = round(out["cuda_cores"]["ms_per_step"] / out["tensor_cores"]["ms_per_step"], 2)
    out["epoch_10k_pairs_s"] = round(10000 / out["tensor_cores"]["pairs_per_s"], 2)
    return out


def batched_section(torch, ops, peak, steps=4):
    """Configuration 5: 512 independent heat problems (cube sides 16..96,
    alpha log-uniform [1e-3, 1e-1], forward or backward Euler, seed 3) in one
    persistent launch per step; tile size and blocks per SM autotuned.  The
    per-member error against an FP64 solve is checked on the 8 smallest
    backward-Euler and 8 smallest forward-Euler members (one step)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    from oracle import oracle as O
    from piro_b200 import workloads as W
    cfg = W.batched()
    B = ops.Batch(cfg["n"], cfg["alpha"], cfg["dt"], cfg["scheme"])
    u0 = W.pack_batch(cfg["fields"], B.offsets, B.total)
    B.set_fields(u0)
    tile, bps = B.autotune()
    schedule = B.schedule()
    # one step from u0 for the error check
    B.set_fields(u0)
    B.step(1)
    one = B.get_fields()
    # timed: `steps` steps (the first pair also captures the graph: run one untimed pair)
    B.set_fields(u0)
    B.step(2)
    B.set_fields(u0)
    ms = B.step(steps) / steps
    info = B.member_info()
    n = cfg["n"].astype(np.int64)
    cells = int((n ** 3).sum())
    be = cfg["scheme"] == 1
    # algorithmic bytes of the last step: forward Euler read u + write out; backward
    # Euler setup 20 B/cell, 40 B/cell per CG iteration, 44 B/cell per residual
    # evaluation (sweeps + 1), the result 4 B/cell
    N = n ** 3
    byt = float((8 * N[~be]).sum()) + float((N[be] * (24 + 40 * info["inner"][be] + 44 * (info["sweeps"][be] + 1))).sum())
    # per-member error against FP64
    errs_be, fe_ok, fe_n = [], 0, 0
    order = np.argsort(n)
    for want, pick in ((True, [k for k in order if be[k]][:8]), (False, [k for k in order if not be[k]][:8])):
        for k in pick:
            m, a, dt = int(n[k]), cfg["alpha"][k], cfg["dt"][k]
            u = cfg["fields"][k]
            got = B.member(one, k)
            if not want:
                ref = O.stencil_fe(m, m, m, dt, u, alpha=np.full(m ** 3, a, np.float32))
                fe_ok += int(np.array_equal(got, ref))
                fe_n += 1
                continue
            idx = np.arange(m ** 3).reshape(m, m, m)
            inter = np.zeros((m, m, m), bool)
            inter[1:-1, 1:-1, 1:-1] = True
            ii = idx[inter]
            c = float(dt) * float(a)
            rows = [ii] + [ii] * 6
            cols = [ii] + [np.roll(idx, -sh, axis=ax)[inter] for ax in range(3) for sh in (-1, 1)]
            vals = [np.full(ii.size, 1.0 + 6.0 * c)] + [np.full(ii.size, -c)] * 6
            A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                              shape=(m ** 3, m ** 3))
            x = u.astype(np.float64)
            x[inter.reshape(-1)] = spla.spsolve(A[inter.reshape(-1)][:, inter.reshape(-1)].tocsc(),
                                                x[inter.reshape(-1)])
            errs_be.append(float(np.abs(got - x).max() / np.abs(x).max()))
    B.close()
    return {
        "members": int(len(n)), "backward_euler_members": int(be.sum()), "cells": cells,
        "ms_per_step": round(ms, 3), "cell_updates_per_s": cells / ms * 1e3,
        "gbs": round(byt / ms / 1e6, 1), "frac": round(byt / ms / 1e6 / peak, 4),
        "autotuned": {"tile_cells": tile, "blocks_per_sm": bps, "schedule": schedule},
        "be_cg_iterations": {"mean": float(info["inner"][be].mean()), "max": int(info["inner"][be].max())},
        "be_sweeps_max": int(info["sweeps"][be].max()),
        "worst_rel_residual": float(info["rel"][be].max()), "all_converged": bool(np.all(info["status"] == 0)),
        "error_vs_fp64": {"be_members_checked": len(errs_be), "be_max_rel_err": max(errs_be) if errs_be else None,
                          "fe_members_bitexact": f"{fe_ok}/{fe_n}"},
        "note": "one cooperative launch per step (two steps per CUDA graph); bytes counted per member from its "
                "CG iterations and refinement sweeps",
    }


# ------------------------------------------------------------------ arms
def fp64_trajectory_check(torch, O, solver, cfg, Ah, x):
    """The configuration's 20 steps from u0 on the device and by the oracle in
    FP64 only; per step the device's FP64 relative residual and the max error
    of its field against the FP64 trajectory (absolute and relative to max |u|)."""
    nx, ny, nz = cfg["n"]
    u = torch.from_numpy(cfg["u0"]).cuda()
    u64 = cfg["u0"].astype(np.float64)
    per = []
    for k in range(cfg["steps"]):
        info = solver.solve(u, x, rtol=1e-8)
        u64, _, rel64 = O.be_cg_f64(nx, ny, nz, Ah, cfg["alpha"], u64, rtol=1e-13)
        got = x.cpu().numpy().astype(np.float64)
        err = float(np.abs(got - u64).max())
        per.append({"step": k + 1, "rel_residual": info.rel_residual, "inner_iterations": info.inner_iterations,
                    "max_abs_err": err, "max_rel_err": err / float(np.abs(u64).max())})
        u, x = x, u
    return {"steps": per, "worst_rel_err": max(p["max_rel_err"] for p in per),
            "worst_rel_residual": max(p["rel_residual"] for p in per),
            "reference": "oracle FP64 Jacobi-PCG to 1e-13 per step (oracle/piro_oracle.c or_be_cg_f64d)"}


def run_piro(args):
    import torch
    import torch.distributed as dist

    from piro_b200 import ops
    from piro_b200 import workloads as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    peak, peak_kind = load_peaks()
    tf_peak = load_tflops_peak()

    cfg = W.heat_be_128()
    nx, ny, nz = cfg["n"]
    N = nx * ny * nz
    A, alpha = be_problem(torch, ops, cfg)
    flush_buf = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")

    def l2_flush():
        flush_buf.zero_()  # a 252 MB write evicts the 126 MB L2
    nnzA = A[2].numel()
    # inner Krylov operator: matrix-free 7-point (checked against A) and CSR
    solver = ops.BESolver(nx, ny, nz, A, alpha, stencil=(float(cfg["dt"]), 1.0))
    solver_csr = ops.BESolver(nx, ny, nz, A, alpha)
    inner_op = solver.inner_operator
    u0 = torch.from_numpy(cfg["u0"]).cuda()
    traj = cfg["steps"]

    def time_steps(sv, steps, warmup, sample_clocks):
        u = u0.clone()
        x = torch.empty_like(u)
        for i in range(warmup):
            if i % traj == 0:
                u.copy_(u0)
            sv.solve(u, x, rtol=1e-8)
            u, x = x, u
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        sv.kernel_stats(reset=True)
        clocks = ClockSampler(local) if sample_clocks else None
        if clocks:
            time.sleep(0.2)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.synchronize()
        iters, outers, worst = [], [], 0.0
        for i in range(steps):
            if i % traj == 0:
                u.copy_(u0)
            l2_flush()  # the step starts with none of its data in L2; outside the step's events
            ev[i][0].record()
            info = sv.solve(u, x, rtol=1e-8)
            ev[i][1].record()
            u, x = x, u
            iters.append(info.inner_iterations)
            outers.append(info.outer_iterations)
            worst = max(worst, info.rel_residual)
        torch.cuda.synchronize()
        ck = clocks.stop() if clocks else None
        ms = sum(a.elapsed_time(b) for a, b in ev) / steps
        pbytes = sv.persistent_bytes()
        nsp, spms, nl = sv.kernel_stats(reset=True)
        if world > 1:
            t = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
            dist.barrier()
        return dict(ms=ms, iters=float(np.mean(iters)), outers=float(np.mean(outers)), worst=worst,
                    spmv_launches=nsp, spmv_ms=spms, launches=nl, clocks=ck, pbytes=pbytes)

    main = time_steps(solver, args.steps, args.warmup, True)
    csr = time_steps(solver_csr, max(10, args.steps // 4), args.warmup, False)
    ms_step = main["ms"]
    ck = main["clocks"]
    x = torch.empty_like(u0)
    # roofline of the dominant kernel (the one persistent launch per step):
    # what binds it is latency -- L2 round trips of the neighbour reads and
    # the grid barriers of each CG iteration -- not HBM (its data stay in L2
    # and shared memory between phases).  achieved/frac: DRAM bytes per launch
    # (the committed ncu capture of the same 128^3 launch) / event-timed
    # duration against the copy peak; binding: the L2-throughput and
    # issue-slot fractions of that capture; effective: the CG bytes of the
    # CSR formulation (8 nnz + 4(N+1) + 60 N per iteration, 8 nnz + 4(N+1) +
    # 24 N per FP64 residual) over the same time.
    k_name = "k_be_persistent" if inner_op == "stencil-persistent" else (
        "k_cg_spmv_mf" if inner_op == "stencil" else "k_cg_spmv")
    avg_spmv_ms = main["spmv_ms"] / max(1, main["spmv_launches"])
    prof = profiled_metrics(k_name)
    traffic = prof.get("traffic_bytes_per_launch")
    dram_gbs = traffic / avg_spmv_ms / 1e6 if traffic else None
    eff_bytes = (main["iters"] * (8 * nnzA + 4 * (N + 1) + 60 * N) +
                 (main["outers"] + 1) * (8 * nnzA + 4 * (N + 1) + 24 * N))
    csr_bytes = 8 * nnzA + 4 * (N + 1) + 20 * N
    csr_avg = csr["spmv_ms"] / max(1, csr["spmv_launches"])
    launches = main["launches"]
    roofline = {
        "kernel": k_name, "bound": "latency",
        "achieved": None if dram_gbs is None else round(dram_gbs, 1), "peak": peak, "unit": "GB/s",
        "frac": None if dram_gbs is None else round(dram_gbs / peak, 4), "peak_kind": peak_kind,
        "traffic": traffic, "avg_launch_ms": avg_spmv_ms, "launches": main["spmv_launches"],
        "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per launch, ncu capture of the same "
                          "128^3 launch (profiles/k_be_persistent_128.md)",
        "binding": {"l2_throughput_frac": (prof["lts__throughput.avg.pct_of_peak_sustained_elapsed"] / 100
                                           if "lts__throughput.avg.pct_of_peak_sustained_elapsed" in prof else None),
                    "issue_active_frac": (prof["smsp__issue_active.avg.pct_of_peak_sustained_active"] / 100
                                          if "smsp__issue_active.avg.pct_of_peak_sustained_active" in prof else None),
                    "us_per_cg_iteration": round(1e3 * avg_spmv_ms / max(main["iters"], 1e-9), 2),
                    "note": "latency bound: L2 round trips of neighbour reads and two grid all-reduces per CG "
                            "iteration; DRAM moves only the step's first touch of its data"},
        "effective": {"bytes_per_launch": eff_bytes, "gbs": round(eff_bytes / avg_spmv_ms / 1e6, 1),
                      "frac_of_hbm_peak": round(eff_bytes / avg_spmv_ms / 1e6 / peak, 4),
                      "note": "algorithmic bytes of the CSR formulation (per CG iteration 8 nnz + 4(N+1) + 60 N, "
                              "per FP64 residual 8 nnz + 4(N+1) + 24 N); this kernel is matrix-free and serves "
                              "them from L2 and shared memory, so the figure exceeds the HBM peak"},
    }

    # end to end through host buffers: every step copies u_n from pinned host
    # memory to the device, solves, and copies u_{n+1} back; the caller then
    # passes the buffer it received as the next input (two pinned buffers
    # ping-pong; the trajectory restarts from u0 every `traj` steps)
    h_u0 = torch.from_numpy(cfg["u0"]).pin_memory()
    hbuf = [torch.empty(N, dtype=torch.float32).pin_memory() for _ in range(2)]
    db = torch.empty_like(u0)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    h_in = h_u0
    fev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        h_out = hbuf[i & 1]
        l2_flush()
        fev[i][0].record()
        db.copy_(h_in, non_blocking=True)
        solver.solve(db, x, rtol=1e-8)
        h_out.copy_(x, non_blocking=True)
        fev[i][1].record()
        torch.cuda.current_stream().synchronize()  # the caller now holds u_{n+1} on the host
        h_in = h_out if (i + 1) % traj else h_u0
    f1.record()
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in fev) / args.steps
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    # the per-configuration sections run on a single-GPU run only: under
    # torchrun the other ranks would wait for them at the closing barrier
    solo = world == 1
    spmv = spmv_section(torch, ops, steps=20, warmup=3, peak=peak) if solo else None
    configs = config_sections(torch, peak) if solo else None
    learned = (learned_section(torch, ops, cfg, A, alpha, ms_step, main["iters"], min(args.steps, 40), tf_peak,
                               l2_flush) if solo else None)
    training = training_section(torch, ops, tf_peak) if solo else None
    batched = batched_section(torch, ops, peak) if solo else None
    next_rows = next_rows_section(torch, ops, peak) if solo else None
    assembly = assembly_section(torch, ops, peak) if solo else None

    cpu = None
    fp64 = None
    if rank == 0 and world == 1:
        from oracle import oracle as O
        Ah = tuple(t.cpu().numpy() for t in A)
        al = cfg["alpha"]
        t0 = time.perf_counter()
        u64, cg_its, rel = O.be_cg_f64(nx, ny, nz, Ah, al, cfg["u0"], rtol=1e-8)
        cpu_ms = (time.perf_counter() - t0) * 1e3
        nthr = O.num_threads()
        O.set_threads(1)
        t0 = time.perf_counter()
        O.be_cg_f64(nx, ny, nz, Ah, al, cfg["u0"], rtol=1e-8)
        cpu1_ms = (time.perf_counter() - t0) * 1e3
        O.set_threads(nthr)
        cpu = {"value": cpu_ms, "unit": "ms/step", "cores": nthr, "kind": "port",
               "sample": f"1 backward-Euler step of the 128^3 config by the oracle's FP64 Jacobi-PCG to 1e-8 "
                         f"({cg_its} iterations), OpenMP over all host threads; a port, no PIRO code runs here "
                         "(PIRO's JLI iteration diverges at this dt)",
               "one_thread": {"value": round(cpu1_ms, 1), "unit": "ms/step", "cores": 1},
               "spmv": spmv.pop("cpu_baseline", None) if spmv else None}
        # per-step error of the device trajectory against an FP64-only one
        # (each step solved to 1e-13 from the previous FP64 solution)
        fp64 = fp64_trajectory_check(torch, O, solver, cfg, Ah, x)

    solver.close()
    solver_csr.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(ms_step, 4), "unit": "ms/step", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 Krylov + f64 refinement", "data": "synthetic (seeded numpy)",
        "config": bench_config(cfg, world),
        "timing": "L2 flushed (a 252 MB write) before every timed step, outside the step's own CUDA-event pair; "
                  "value and e2e are sums of per-step event times",
        "solver": {"inner_operator": inner_op, "preconditioner": "jacobi",
                   "inner_iterations_mean": main["iters"],
                   "outer_sweeps_mean": main["outers"], "worst_rel_residual": main["worst"],
                   "csr_inner_operator": {"ms_per_step": round(csr["ms"], 4), "inner_iterations_mean": csr["iters"],
                                          "worst_rel_residual": csr["worst"], "k_cg_spmv_avg_ms": csr_avg,
                                          "k_cg_spmv_gbs": round(csr_bytes / csr_avg / 1e6, 1)}},
        "roofline": roofline,
        "e2e": {"value": round(e2e_ms, 4), "unit": "ms/step", "h2d_bytes_per_step": 4 * N, "d2h_bytes_per_step": 4 * N},
        "gpu_launches": launches,
        "clocks": ck,
        "spmv_256": spmv,
        "configs": configs,
        "learned": learned,
        "training": training,
        "batched": batched,
        "next_rows": next_rows,
        "assembly": assembly,
        "fp64_check": fp64,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_reference(args):
    """CPU arm: the oracle's FP64 Jacobi-PCG (the reference's own JLI diverges
    at this dt) on the same 128^3 step, all host threads, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    from piro_b200 import workloads as W
    cfg = W.heat_be_128()
    nx, ny, nz = cfg["n"]
    N = nx * ny * nz
    L = O.laplacian(nx, ny, nz, 3, np.float32(1.0))
    Ls = (L[0], L[1], O.csr_rowscale(N, L[0], L[2], cfg["alpha"]))
    I = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.float32))
    A = O.csrgeam2(N, I, np.float32(-cfg["dt"]), Ls)
    u = cfg["u0"].copy()
    times = []
    for i in range(args.warmup + args.steps):
        if i % cfg["steps"] == 0:
            u = cfg["u0"].copy()
        t0 = time.perf_counter()
        u64, _, _ = O.be_cg_f64(nx, ny, nz, A, cfg["alpha"], u, rtol=1e-8)
        dt_ms = (time.perf_counter() - t0) * 1e3
        u = u64.astype(np.float32)
        if i >= args.warmup:
            times.append(dt_ms)
    v = float(np.mean(times))
    line = {
        "metric": METRIC, "value": round(v, 3), "unit": "ms/step", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded numpy)", "impl": "reference",
        "config": bench_config(cfg, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": round(v, 3), "unit": "ms/step", "cores": O.num_threads(), "kind": "port",
                         "sample": "each step one full backward-Euler solve by the oracle's FP64 Jacobi-PCG "
                                   "(OpenMP, all host threads); a port of the method, no PIRO code runs in this "
                                   "arm, because PIRO's own JLI iteration diverges at this dt"},
        "e2e": {"value": round(v, 3), "unit": "ms/step", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_sharded(args):
    """One grid over all ranks: the backward-Euler configuration's family at
    256^3 (smoothed log-normal alpha, sigma 1.5, filter 8, seed 2; dt = 50x
    the explicit limit) split into z-slabs, one per GPU
    (piro_b200/slab.py SlabBE: halo planes and FP64 sums over NCCL, the CG
    scalars kept on the device and the done flag read every 8 iterations).
    A step is one backward-Euler solve to a 1e-8 FP64 relative residual, the
    next step starting from its result; strong scaling (the grid is fixed)."""
    import datetime

    import torch
    import torch.distributed as dist

    from piro_b200 import slab
    from piro_b200 import workloads as W
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        comm = slab.TorchComm()
    else:
        comm = slab.LocalComm(slab.LocalGroup(1), 0)
    n = args.sharded
    cfg = W.heat_be_128(n=n)
    nx = ny = nz = n
    plane = nx * ny
    z0, z1 = slab.split_planes(nz, world)[rank]
    lo, hi = (z0 - 1) * plane, (z1 + 1) * plane

    def local_of(full):
        out = np.zeros(hi - lo, np.float32)
        s0, s1 = max(lo, 0), min(hi, nx * ny * nz)
        out[s0 - lo:s1 - lo] = full[s0:s1]
        return torch.from_numpy(out).cuda()
    be = slab.CudaBackend()
    sv = slab.SlabBE(be, comm, nx, ny, nz, z0, z1, float(cfg["dt"]), 1.0, local_of(cfg["alpha"]))
    b0 = local_of(cfg["u0"])
    b = b0.clone()
    traj = cfg["steps"]
    iters = []

    def step():
        x64, info = sv.solve(b, rtol=1e-8, device_scalars=True, check_every=8)
        if info["status"] != "ok":
            raise RuntimeError(f"sharded solve: {info}")
        iters.append(info["inner"])
        b.copy_(x64.float())
    for i in range(args.warmup):
        if i % traj == 0:
            b.copy_(b0)
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    iters.clear()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        if i % traj == 0:
            b.copy_(b0)
        ev[i][0].record()
        step()
        ev[i][1].record()
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(c) for a, c in ev) / args.steps
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": f"BE {n}^3 step ms at 1e-8 FP64 residual, one grid in z-slabs over {world} GPU(s)",
        "value": round(ms, 4), "unit": "ms/step", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 Krylov + f64 refinement", "data": "synthetic (seeded numpy)",
        "config": {"workload": f"heat backward Euler {n}^3, smoothed log-normal alpha (sigma 1.5, filter 8, seed 2), "
                               "dt = 50x explicit limit", "grid": [nx, ny, nz], "parallelism": f"z-slab x{world}",
                   "slab_planes": [z1 - z0 for z0, z1 in slab.split_planes(nz, world)]},
        "solver": {"inner_iterations_mean": float(np.mean(iters)) if iters else None,
                   "scalars": "on the device (all-reduced sums read by the next kernel), done flag read every 8 "
                              "iterations"},
    }
    print(json.dumps(line), flush=True)


def run_profile_case(args):
    """Small fixed cases for ncu captures (no timing, no JSON): `be` solves the
    128^3 backward-Euler step twice, `spmv` runs the 256^3 forward-Euler
    kernels (CSR, matrix-free, fused CSR + setBC, indexed COO; about 1.5 GB
    on the device), `dense` three DENSE steps at N = 12,288 (a 604 MB
    matrix), `learned` two learned-preconditioner solves of the 128^3 step,
    `batched` two steps of a 64-member batch
    in each schedule (lockstep, then grouped), `train` four training steps of
    the network on 8 crops of 34^3 cells, `ht` three staged and three one-pass
    ordered hash-table steps at 192^3, `fe160` the forward-Euler kernels one format at a time at 160^3
    (CSR, matrix-free, segmented COO, three launches each), three
    Laplacian assemblies and three v.grad merges (csrgeam3) of the upwind
    gradients, `lu` the scheme-27 band factorization and one solve at 24^3."""
    import torch

    from piro_b200 import ops
    from piro_b200 import workloads as W
    torch.cuda.set_device(0)
    if args.profile == "be":
        cfg = W.heat_be_128()
        nx, ny, nz = cfg["n"]
        A, alpha = be_problem(torch, ops, cfg)
        s = ops.BESolver(nx, ny, nz, A, alpha, stencil=(float(cfg["dt"]), 1.0))
        b = torch.from_numpy(cfg["u0"]).cuda()
        x = torch.empty_like(b)
        for _ in range(2):
            info = s.solve(b, x, rtol=1e-8)
        print("be", s.inner_operator, info.inner_iterations, info.rel_residual)
        s.close()
    elif args.profile == "dense":
        A = ops.dense_laplacian(32, 24, 16, 3, 1.0)
        u = torch.rand(32 * 24 * 16, device="cuda")
        x = torch.empty_like(u)
        for _ in range(3):
            ops.dense_fe_step(A, 0.01, u, x)
        ops.dense_check()
        print("dense ok")
    elif args.profile == "learned":
        cfg = W.heat_be_128()
        nx, ny, nz = cfg["n"]
        A, alpha = be_problem(torch, ops, cfg)
        net = ops.PCNet(seed=0)
        net.set_params(np.load(os.path.join(ROOT, "piro_b200", "data", "pcnet_be128.npy")))
        s = ops.BESolver(nx, ny, nz, A, alpha, stencil=(float(cfg["dt"]), 1.0))
        s.set_preconditioner(net)
        b = torch.from_numpy(cfg["u0"]).cuda()
        x = torch.empty_like(b)
        for _ in range(2):
            info = s.solve(b, x, rtol=1e-8)
        print("learned", info.inner_iterations, info.rel_residual)
        s.close()
        net.close()
    elif args.profile == "ht":
        n = 192  # 7.1M rows, a 0.85 GB table: larger than L2, small enough to capture
        N = n ** 3
        A = ops.csr_laplacian(n, n, n, 3, 1.0)
        ts = ops.ht_table_size(A[2].numel(), N, 1)
        keys, vals = ops.ht_build(N, *A, ts)
        del A
        order = ops.ht_row_order(N, ts)
        u = torch.rand(N, device="cuda")
        out = torch.empty_like(u)
        stage = ops.ht_stage(N)
        for _ in range(3):
            ops.ht_spmv_staged(n, n, n, keys, vals, 0.01, order, stage, u, out, fe=True)
        for _ in range(3):
            ops.ht_spmv_ordered(n, n, n, keys, vals, 0.01, order, u, out, fe=True)
        torch.cuda.synchronize()
        print("ht ok", ts)
    elif args.profile == "train":
        m, batch = 34, 8
        N = m ** 3
        rng = np.random.default_rng(5)
        r, f, t = (torch.from_numpy(rng.standard_normal(batch * N).astype(np.float32)).cuda() for _ in range(3))
        mk = torch.ones(batch * N, device="cuda")
        net = ops.PCNet(seed=0)
        for _ in range(3):
            net.loss_grad(m, m, m, r, f, t, mk, batch=batch, want_loss=False)
            net.adam_step(1e-4)
        loss, _ = net.loss_grad(m, m, m, r, f, t, mk, batch=batch)
        print("train", loss)
        net.close()
    elif args.profile == "batched":
        cfg = W.batched(count=64)
        B = ops.Batch(cfg["n"], cfg["alpha"], cfg["dt"], cfg["scheme"])
        u0 = W.pack_batch(cfg["fields"], B.offsets, B.total)
        for grouped in (False, True):
            B.set_schedule(grouped, 4)
            B.set_fields(u0)
            B.step(2)
        print("batched ok")
    elif args.profile == "lu":
        n = 24  # N = 13,824, bandwidth 576: a 191 MB band, larger than L2
        N = n ** 3
        L = ops.csr_laplacian(n, n, n, 3, 1.0)
        ts = ops.ht_table_size(L[2].numel(), N, 1)
        keys, vals = ops.ht_build(N, *L, ts)
        lu = ops.HtLu(N, n * n, keys, vals, ts, 1.0, -0.05)
        b = torch.rand(N, device="cuda")
        lu.solve(b)
        torch.cuda.synchronize()
        print("lu ok")
    elif args.profile == "fe160":
        cfg = W.spmv_256(n=160)  # 4.1M rows, 28.4M nonzeros: above L2, well under a GB
        nx, ny, nz = cfg["n"]
        N = nx * ny * nz
        u = torch.from_numpy(cfg["u"]).cuda()
        alpha = torch.from_numpy(cfg["alpha"]).cuda()
        out = torch.empty_like(u)
        A = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
        ops.csr_rowscale(A[0], A[2], alpha)
        for _ in range(3):
            ops.csr_fe_step(nx, ny, nz, A, 0.01, u, out)
        for _ in range(3):
            ops.stencil_fe_step(nx, ny, nz, 0.01, u, out, alpha=alpha)
        rows = torch.repeat_interleave(torch.arange(N, device="cuda", dtype=torch.int32),
                                       (A[0][1:] - A[0][:-1]).to(torch.int64))
        for _ in range(3):
            ops.coo_spmv(N, (rows, A[1], A[2]), 0.01, u, out, fe=True)
        for _ in range(3):
            ops.csr_laplacian(nx, ny, nz, 3, 1.0)
        del A, rows
        G = [ops.csr_gradient(nx, ny, nz, 1, a, 2.0) for a in range(3)]
        v = torch.rand(3 * N, device="cuda")
        for _ in range(3):
            ops.csrgeam3(N, *G, v)
        torch.cuda.synchronize()
        print("fe160 ok")
    else:
        cfg = W.spmv_256()
        nx, ny, nz = cfg["n"]
        u = torch.from_numpy(cfg["u"]).cuda()
        alpha = torch.from_numpy(cfg["alpha"]).cuda()
        out = torch.empty_like(u)
        A = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
        ops.csr_rowscale(A[0], A[2], alpha)
        for _ in range(4):
            ops.csr_fe_step(nx, ny, nz, A, 0.01, u, out)
        for _ in range(4):
            ops.stencil_fe_step(nx, ny, nz, 0.01, u, out, alpha=alpha)
        for _ in range(2):
            ops.csr_fe_step_bc(nx, ny, nz, A, 0.01, u, u, out)
        N = nx * ny * nz
        rows = torch.repeat_interleave(torch.arange(N, device="cuda", dtype=torch.int32),
                                       (A[0][1:] - A[0][:-1]).to(torch.int64))
        rowstart = ops.coo_row_index(N, rows)
        for _ in range(2):
            ops.coo_step_indexed(N, rowstart, A[1], A[2], 0.01, u, out, fe=True)
        del rows, rowstart
        torch.cuda.synchronize()
        print("spmv ok")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="piro", choices=["piro", "reference"])
    ap.add_argument("--sharded", type=int, default=0, metavar="N",
                    help="one N^3 backward-Euler grid in z-slabs over the ranks (strong scaling) instead of replicas")
    ap.add_argument("--profile", choices=["be", "spmv", "fe160", "lu", "dense", "learned", "batched", "train", "ht"],
                    help="run a small fixed case for ncu, print no JSON")
    args = ap.parse_args()
    if args.profile:
        run_profile_case(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.sharded:
        run_sharded(args)
    else:
        run_piro(args)


if __name__ == "__main__":
    main()
