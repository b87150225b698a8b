#!/usr/bin/env python3
"""Headline benchmark: FCG + BCMG (suitor matching, pairwise aggregation AMG) set-up + solve to
relative residual 1e-8 on the 27-point 3D Poisson problem on 160^3 (4,096,000 rows,
109,215,352 non-zeros, FP64 CSR; x* uniform[-1,1] from numpy default_rng(1), b = A x*).

One step = hierarchy set-up + FCG solve with the FP32 V-cycle inside FP64 FCG, inputs resident
in HBM. The same step with the plain FP64 V-cycle, the fine-level SpMV bandwidth, per-kernel
roofline figures, the end-to-end time through the C ABI with host buffers, and a CPU baseline
(the OpenMP restatement of the same method, on this host's cores) are reported beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Multi-GPU (torchrun, one process per GPU): each rank solves its own copy of the system
(independent replicas, no collective on the data path); time = max over ranks. The batched
forms shard instead: rank r takes systems r, r + N, ... of the 256 (--batch) and a contiguous
slice of the 32 right-hand-side columns (--multi).
--impl reference times the reference algorithm's CPU restatement (oracle/, OpenMP) on rank 0.
"""
from __future__ import annotations

import os
import sys

# The host cores this process may run on, read before any OpenMP runtime loads: with thread
# binding on, libgomp pins the calling thread to one core when it starts.
HOST_CPUS = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
# The CPU legs (the reference arm, and the CPU baseline, which runs in a child process) pin their
# OpenMP threads one per core; the GPU arm leaves its host threads unpinned.
PIN_ENV = {"OMP_PROC_BIND": "close", "OMP_PLACES": "cores"}
if "--impl=reference" in sys.argv or "--cpu-leg" in sys.argv or (
        "--impl" in sys.argv and sys.argv[sys.argv.index("--impl") + 1:][:1] == ["reference"]):
    for _k, _v in PIN_ENV.items():
        os.environ.setdefault(_k, _v)

import argparse
import datetime
import json
import statistics
import subprocess
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FCG+AMG setup+solve s to rel-res 1e-8, FP32-Vcycle vs FP64; SpMV HBM GB/s"
WORKLOADS = {
    "poisson27_160": {"stencil": 27, "grid": (160, 160, 160), "seed": 1,
                      "text": "3D Poisson 27-point 160^3 Dirichlet (diag 26, off -1), FP64 CSR"},
    "poisson7_50": {"stencil": 7, "grid": (50, 50, 50), "seed": 0,
                    "text": "3D Poisson 7-point 50^3 Dirichlet (diag 6, off -1), FP64 CSR"},
    "poisson27_100": {"stencil": 27, "grid": (100, 100, 100), "seed": 1,
                      "text": "3D Poisson 27-point 100^3 Dirichlet, FP64 CSR"},
    "diffusion7_256": {"kind": "diffusion", "grid": (256, 256, 256), "theta_seed": 2, "rhs_seed": 3,
                       "text": "7-point FV diffusion 256^3, kappa = exp(theta), theta Gaussian random field "
                               "(squared-exponential, length 8, sigma 2, seed 2), harmonic-mean faces; b ~ U[0,1] (seed 3)"},
    "diffusion7_64": {"kind": "diffusion", "grid": (64, 64, 64), "theta_seed": 2, "rhs_seed": 3,
                      "text": "7-point FV diffusion 64^3 (small variant of diffusion7_256)"},
}
ADJOINT = {"grid": (96, 96, 96), "theta_seed": 5, "noise_seed": 6, "directions": 20, "step": 1e-6, "rtol": 1e-10}
RTOL = 1e-8
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return PEAKS_FALLBACK["hbm_gbs"], "fallback"


def build_problem(wl):
    import scipy.sparse as sp
    import bootcmatchgx_b200 as bx
    if wl.get("kind") == "diffusion":
        from bootcmatchgx_b200 import problems
        g = wl["grid"]
        theta = problems.gaussian_random_field(g, length=8.0, sigma=2.0, seed=wl["theta_seed"])
        row, col, val = bx.diffusion_7p(*g, np.exp(theta).reshape(-1, order="F").reshape(-1))
        b = np.random.default_rng(wl["rhs_seed"]).uniform(0.0, 1.0, row.size - 1)
        return row, col, val, None, b
    st, (nx, ny, nz), seed = wl["stencil"], wl["grid"], wl["seed"]
    row, col, val = bx.laplacian_3d(st, nx, ny, nz)
    n = row.size - 1
    xs = np.random.default_rng(seed).uniform(-1.0, 1.0, n)
    b = sp.csr_matrix((val, col, row), shape=(n, n)) @ xs
    return row, col, val, xs, b


# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # nvidia-smi's start-up (driver initialisation) competes with the host side of the set-up:
        # the timed region begins once its first sample is written
        t0 = time.time()
        while time.time() - t0 < 1.5 and os.path.getsize(self.f.name) == 0 and self.proc.poll() is None:
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [l.strip().split(", ") for l in self.f.read().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
def host_info():
    """CPU model and CPU counts of this host (/proc/cpuinfo; lscpu need not be installed)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "logical_cpus": os.cpu_count(), "cpus_available": HOST_CPUS,
            "omp_proc_bind": os.environ.get("OMP_PROC_BIND"), "omp_places": os.environ.get("OMP_PLACES")}


def diffusion_csr_numpy(nx, ny, nz, kappa):
    """The 7-point FV diffusion matrix in numpy, with bcmgx_diffusion_7p's arithmetic and order
    (cells x fastest, columns ascending, the diagonal summed over the faces -z, -y, -x, +x, +y,
    +z): the reference arm builds its matrix without the product library."""
    N = nx * ny * nz
    r = np.arange(N)
    gi, gj, gk = r % nx, (r // nx) % ny, r // (nx * ny)
    k = np.asarray(kappa, dtype=np.float64).reshape(-1)
    faces = [(0, 0, -1), (0, -1, 0), (-1, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)]
    cols = np.full((N, 7), -1, np.int64)
    vals = np.zeros((N, 7))
    diag = np.zeros(N)
    for t, (dx, dy, dz) in enumerate(faces):
        slot = t if t < 3 else t + 1
        a, b_, c = gi + dx, gj + dy, gk + dz
        inside = (a >= 0) & (a < nx) & (b_ >= 0) & (b_ < ny) & (c >= 0) & (c < nz)
        j = np.where(inside, a + nx * (b_ + ny * c), 0)
        kj = k[j]
        tij = 2.0 * k * kj / (k + kj)
        diag = diag + np.where(inside, tij, 2.0 * k)
        cols[inside, slot] = j[inside]
        vals[inside, slot] = -tij[inside]
    cols[:, 3] = r
    vals[:, 3] = diag
    keep = cols >= 0
    row = np.zeros(N + 1, np.int32)
    row[1:] = np.cumsum(keep.sum(axis=1))
    return row, cols[keep].astype(np.int32), vals[keep]


def oracle_problem(wl):
    """The workload built without the product library: the Laplacians by the oracle's generator
    (the reference's row order) with b = A x* by the oracle's SpMV; the diffusion matrix by
    diffusion_csr_numpy. Returns (oracle matrix, x* or None, b)."""
    from oracle import pyoracle as O
    if wl.get("kind") == "diffusion":
        from bootcmatchgx_b200 import problems   # numpy only: loads no shared library
        g = wl["grid"]
        theta = problems.gaussian_random_field(g, length=8.0, sigma=2.0, seed=wl["theta_seed"])
        row, col, val = diffusion_csr_numpy(*g, np.exp(theta).reshape(-1, order="F"))
        b = np.random.default_rng(wl["rhs_seed"]).uniform(0.0, 1.0, row.size - 1)
        return O.Matrix.from_csr(row, col, val), None, b
    A = O.Matrix.lap3d(wl["stencil"], *wl["grid"])
    n = A.info()[0]
    xs = np.random.default_rng(wl["seed"]).uniform(-1.0, 1.0, n)
    return A, xs, A.spmv(xs)


def oracle_solve(O, A, b, rtol=RTOL):
    """One full set-up + FCG solve by the oracle; returns (set-up s, solve s, x, info, levels)."""
    t0 = time.perf_counter()
    H = O.Hierarchy(A, O.params(rtol=rtol))
    t1 = time.perf_counter()
    x, info = H.solve(b)
    t2 = time.perf_counter()
    return t1 - t0, t2 - t1, x, info, H.level_sizes()


def cpu_baseline_leg(wl, runs=5):
    """The oracle (OpenMP C++ restatement of the same FCG+BCMG method) on this host's cores,
    threads pinned one per core: `runs` full set-up + solve runs of the same workload, the
    median reported. Also returns the oracle's solution and level sizes for the parity check."""
    from oracle import pyoracle as O
    hi = host_info()
    cores = hi["cpus_available"]
    O.num_threads(cores)
    A, xs, b = oracle_problem(wl)
    runs_out = [oracle_solve(O, A, b) for _ in range(runs)]
    tot = [r[0] + r[1] for r in runs_out]
    med = sorted(range(runs), key=lambda i: tot[i])[runs // 2]
    ts, tv, x, info, levels = runs_out[med]
    line = {"value": tot[med], "unit": "s", "cores": cores, "kind": "port",
            "sample": f"median of {runs} full set-up + full FCG solve runs ({info['niter']} iterations) of "
                      f"the same workload with oracle/bcmgx_oracle.cpp, OMP threads={cores} pinned one per core",
            "runs_s": tot, "setup_s": ts, "solve_s": tv, "niter": info["niter"], "host": hi,
            "err_vs_xstar": None if xs is None else float(np.linalg.norm(x - xs) / np.linalg.norm(xs))}
    return line, {"x": x, "niter": info["niter"], "levels": levels}


def cpu_baseline(workload, runs=5):
    """cpu_baseline_leg in a child process (python bench.py --cpu-leg), so that its OpenMP threads
    are pinned without pinning the GPU arm's host threads; its results come back through a file."""
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "leg.npz")
        env = dict(os.environ, **PIN_ENV)
        subprocess.run([sys.executable, os.path.abspath(__file__), "--cpu-leg", out, "--workload", workload,
                        "--steps", str(runs)], check=True, env=env)
        z = np.load(out, allow_pickle=False)
        line = json.loads(str(z["line"]))
        return line, {"x": z["x"], "niter": int(z["niter"]), "levels": [tuple(t) for t in z["levels"].tolist()]}


def reference_arm(a, wl, rank, world):
    """--impl reference: the reference algorithm on the host cores (the reference itself has no
    CPU implementation, and its CUDA build needs MPI; the oracle port stands in). Every step,
    warm-ups included, is one full set-up + FCG solve to 1e-8; nothing is extrapolated. The
    problem is built by the oracle's own generator, so this arm loads no product code."""
    if rank != 0:
        return None
    from oracle import pyoracle as O
    hi = host_info()
    cores = hi["cpus_available"]
    O.num_threads(cores)
    A, xs, b = oracle_problem(wl)
    n, _, nnz = A.info()
    times, niter = [], None
    for step in range(a.warmup + a.steps):
        ts, tv, x, info, _ = oracle_solve(O, A, b)
        niter = info["niter"]
        if step >= a.warmup:
            times.append(ts + tv)
    v = float(np.mean(times))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": a.workload, "problem": wl["text"], "rtol": RTOL, "rows": int(n), "nnz": int(nnz)},
            "median_s": float(np.median(times)), "niter": niter,
            "cpu_baseline": {"value": v, "unit": "s", "cores": cores, "kind": "port", "host": hi,
                             "sample": "oracle/bcmgx_oracle.cpp (OpenMP restatement of FCG+BCMG, threads pinned one "
                                       f"per core): every step a full set-up + FCG solve to 1e-8 ({niter} iterations)"},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


# ---------------------------------------------------------------------------------------------
def max_over_ranks(x, world, device=None):
    """The largest value of x over all ranks of the job (a time is reported as the slowest rank's);
    x itself when the job has one rank. Works on any process-group backend (NCCL, gloo)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_vcycle(h, r, stream, reps=10):
    """ms of one preconditioner application v = B r (the V-cycle) on device vectors, CUDA events
    on the hierarchy's stream, after one warm-up application."""
    import torch
    h.prec_apply(r)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        h.prec_apply(r)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def vcycle_bytes(inf, pre, post, coarse):
    """Algorithmic bytes of one FP32 V-cycle as the kernels run it: on every level but the last,
    pre + post - 1 l1-Jacobi sweeps over the FP32 matrix (the first pre-sweep starts from zero and
    reads no matrix), the residual, the restriction R r (one entry per fine row) and the
    prolongation x += p x_c[agg]; the coarsest level runs `coarse` FP64 sweeps (the first from
    zero). Matrix entries
    count index_bytes + value bytes (1 where the level streams 1-byte value codes, else 4; 8 for the
    coarsest level's FP64 values; index_bytes 0, pattern-indexed rows, streams 1 byte per row instead),
    vectors 4 bytes (8 on the coarsest level); level 0 also reads the FP64 residual and writes the FP64
    output."""
    n, z, ib = inf["n"], inf["nnz"], inf["index_bytes"]
    vb = [1 if c else 4 for c in inf["value_codes"]]
    total = 0
    for l in range(len(n) - 1):
        nl, zl, nc = n[l], z[l], n[l + 1]
        mat = (ib[l] + vb[l]) * zl + (nl if ib[l] == 0 else 0)
        sweep = mat + 4 * (nl + 1) + 16 * nl
        total += (pre + post - 1) * sweep + 12 * nl
        total += mat + 4 * (nl + 1) + 12 * nl
        total += 4 * (nc + 1) + 8 * nl + 4 * nl + 4 * nc
        total += 8 * nl + 4 * nc + 8 * nl
        if l == 0:
            total += 8 * nl + 4 * nl
    nL, zL = n[-1], z[-1]
    total += (coarse - 1) * ((ib[-1] + (1 if inf["value_codes"][-1] else 8)) * zL + (nL if ib[-1] == 0 else 0)
                             + 4 * (nL + 1) + 32 * nL) + 24 * nL
    return int(total)


def vcycle_roofline(ms, inf, p, peak, peak_kind):
    b = vcycle_bytes(inf, p.prerelax_sweeps, p.postrelax_sweeps, p.relaxnumber_coarse)
    return {"ms": ms, "algorithmic_bytes": b, "gbs": b / ms / 1e6, "frac": b / ms / 1e6 / peak,
            "peak": peak, "peak_kind": f"{peak_kind} hbm_gbs (copy)",
            "what": "one FP32 V-cycle (bcmgx_prec_apply on device vectors), CUDA events"}


def run_ours(a, wl, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import bootcmatchgx_b200 as bx
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    row, col, val, xs, b = build_problem(wl)
    n, nnz = row.size - 1, col.size
    d_row = torch.from_numpy(row).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_val = torch.from_numpy(val).to(dev)
    d_b = torch.from_numpy(b).to(dev)
    d_x = torch.zeros(n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    launches0 = bx.lib().bcmgx_launch_count()

    def params(prec, **kw):
        base = dict(solver="FCG", preconditioner="BCMG", rtol=RTOL, dispnorm=0,
                    vcycle_precision=prec, stream=stream.cuda_stream)
        base.update(kw)
        return bx.params_default(**base)

    def step(prec, keep=False):
        h = bx.Hierarchy(d_row, d_col, d_val, params(prec))
        d_x.zero_()
        _, info = h.solve(d_b, d_x)
        inf = h.info()
        if keep:
            return h, info, inf
        h.free()
        return None, info, inf

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(prec, steps):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0 = bx.lib().bcmgx_launch_count()
        e0.record(stream)
        infos = []
        for _ in range(steps):
            infos.append(step(prec)[1:])
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps, world, dev)
        launches = (bx.lib().bcmgx_launch_count() - c0) / steps
        return ms, infos, launches

    # ---- cold first calls: the first set-up of each form in this process runs the threads-per-row
    # autotuner (its choices are then cached per matrix shape) and loads the kernels
    cold = {}
    for prec in ("FP32", "FP64"):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, info0, inf0 = step(prec)
        torch.cuda.synchronize()
        cold[prec.lower()] = {"setup_ms": inf0["setup_ms"], "solve_ms": info0["solve_ms"],
                              "wall_ms": (time.perf_counter() - t0) * 1e3}
    # ---- headline: FP32 V-cycle inside FP64 FCG
    clocks = ClockSampler(local_rank)
    clocks.start()
    for _ in range(max(0, a.warmup - 1)):
        step("FP32")
    ms32, infos32, launches32 = timed("FP32", a.steps)
    clk = clocks.stop()
    x32 = d_x.cpu().numpy().copy()
    # ---- plain FP64 form (same step, FP64 V-cycle)
    k64 = max(1, min(a.steps, 3))
    for _ in range(max(0, a.warmup - 1)):
        step("FP64")
    ms64, infos64, _ = timed("FP64", k64)
    x64 = d_x.cpu().numpy().copy()
    # ---- tight FP64 oracle solution (rtol 1e-12) for the error statements
    h_t = bx.Hierarchy(d_row, d_col, d_val, params("FP64", rtol=1e-12))
    d_x.zero_()
    h_t.solve(d_b, d_x)
    xt = d_x.cpu().numpy().copy()
    h_t.free()

    # ---- kernel figures on kept hierarchies (same stream, CUDA events)
    h32, _, inf32 = step("FP32", keep=True)
    k32 = h32.time_kernels(0, reps=20)
    vc_ms = time_vcycle(h32, d_b, stream)
    h64, _, inf64 = step("FP64", keep=True)
    k64f = h64.time_kernels(0, reps=20)
    spmv_ms = k64f["spmv"]
    lvl = [h32.time_kernels(l, reps=10) for l in range(1, inf32["num_levels"])]
    h32.free()
    h64.free()
    peak, peak_kind = read_peaks()
    # algorithmic bytes of the format the kernels stream: int16 column offsets (2 B) where the
    # level has them, else int32 (4 B), or with pattern-indexed rows (index bytes 0) one byte per
    # row naming its offsets; 1-byte value codes where the level has them, else the 4- or 8-byte
    # values; bcmgx_spmv on raw CSR arrays always streams int32 + FP64
    ib32, ib64 = inf32["index_bytes"][0], inf64["index_bytes"][0]
    vb32 = 1 if inf32["value_codes"][0] else 4
    vb64 = 1 if inf64["value_codes"][0] else 8
    rb32, rb64 = (n if ib32 == 0 else 0), (n if ib64 == 0 else 0)
    bytes_spmv = 12 * nnz + 4 * (n + 1) + 16 * n
    bytes_jac32 = (ib32 + vb32) * nnz + rb32 + 4 * (n + 1) + 16 * n
    bytes_jac64 = (ib64 + vb64) * nnz + rb64 + 4 * (n + 1) + 32 * n
    bytes_jac32_csr = 8 * nnz + 4 * (n + 1) + 16 * n   # the same sweep on int32 columns + FP32 values
    gbs_spmv = bytes_spmv / (spmv_ms * 1e-3) / 1e9
    gbs_jac32 = bytes_jac32 / (k32["jacobi"] * 1e-3) / 1e9
    gbs_jac64 = bytes_jac64 / (k64f["jacobi"] * 1e-3) / 1e9

    # ---- end to end through the C ABI with host buffers (pinned), FP32 V-cycle
    p_row = torch.from_numpy(row).pin_memory()
    p_col = torch.from_numpy(col).pin_memory()
    p_val = torch.from_numpy(val).pin_memory()
    p_b = torch.from_numpy(b).pin_memory()
    p_x = torch.zeros(n, dtype=torch.float64).pin_memory()
    ke = max(1, min(a.steps, 3))

    def e2e_step():
        h = bx.Hierarchy(p_row.numpy(), p_col.numpy(), p_val.numpy(), params("FP32"))
        p_x.zero_()
        xh, info = h.solve(p_b.numpy(), p_x.numpy())
        h.free()
        return xh, info

    e2e_step()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(ke):
        xh, _ = e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / ke
    e2e_ms = max_over_ranks(max(e0.elapsed_time(e1) / ke, wall * 1e3), world, dev)

    if rank != 0:
        return None, None
    setup32 = float(np.mean([i[1]["setup_ms"] for i in infos32]))
    solve32 = float(np.mean([i[0]["solve_ms"] for i in infos32]))
    setup64 = float(np.mean([i[1]["setup_ms"] for i in infos64]))
    solve64 = float(np.mean([i[0]["solve_ms"] for i in infos64]))
    nrm = np.linalg.norm
    tpr0 = inf32["tpr"][0]   # level 0's kernel code: threads per row, negative staged, 64 sliced
    form0 = "sliced" if tpr0 == 64 else "staged" if tpr0 < 0 else "plain"
    kname0 = {"sliced": "k_rowop_sliced<", "staged": f"k_rowop_staged<{-tpr0},", "plain": f"k_rowop<{tpr0},"}[form0]
    line = {
        "metric": METRIC, "value": ms32 / 1e3, "unit": "s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms32, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 outer FCG / f32 V-cycle", "data": "synthetic",
        "config": {"workload": a.workload, "problem": wl["text"], "rows": int(n), "nnz": int(nnz),
                   "rhs": (f"b = A x*, x* ~ U[-1,1] (numpy default_rng({wl['seed']}))" if xs is not None
                           else f"b ~ U[0,1] (numpy default_rng({wl['rhs_seed']}))"),
                   "rtol": RTOL, "settings": "FCG_BCMG.properties defaults (aggrsweeps 2, 4+4 l1-Jacobi, "
                   "20 coarse sweeps, V-cycle)", "vcycle": "fp32",
                   "l2": "inputs larger than L2 (CSR 1.39 GB)" if nnz > 5e7 else "inputs fit in L2",
                   "parallelism": f"replicas x{world} (one independent system per GPU)"},
        "breakdown": {"setup_ms": setup32, "solve_ms": solve32, "niter": infos32[-1][0]["niter"],
                      "threads_per_row": inf32["tpr"], "index_bytes": inf32["index_bytes"],
                      "value_codes": inf32["value_codes"],
                      "levels": inf32["n"], "level_nnz": inf32["nnz"], "op_cmplx": inf32["op_cmplx"]},
        "fp64": {"value": ms64 / 1e3, "setup_ms": setup64, "solve_ms": solve64,
                 "niter": infos64[-1][0]["niter"]},
        "fp32_speedup_vs_fp64": ms64 / ms32,
        "errors": {"fp32_vs_xstar": None if xs is None else float(nrm(x32 - xs) / nrm(xs)),
                   "fp64_vs_xstar": None if xs is None else float(nrm(x64 - xs) / nrm(xs)),
                   "fp32_vs_fp64_tight": float(nrm(x32 - xt) / nrm(xt)),
                   "fp64_vs_fp64_tight": float(nrm(x64 - xt) / nrm(xt)),
                   "fp32_vs_fp64": float(nrm(x32 - x64) / nrm(x64)),
                   "fp32_rel_residual": float(nrm(b - _spmv(row, col, val, x32)) / nrm(b))},
        "spmv": {"gbs": gbs_spmv, "ms": spmv_ms, "bytes": bytes_spmv, "frac_of_peak": gbs_spmv / peak,
                 "frac_of_8TBs_nominal": gbs_spmv / 8000.0},
        "kernels_level0": {"index_bytes": ib32, "value_bytes_fp32": vb32, "value_bytes_fp64": vb64,
                           "fp32_jacobi_ms": k32["jacobi"], "fp32_jacobi_gbs": gbs_jac32,
                           "fp32_jacobi_csr_equivalent_gbs": bytes_jac32_csr / (k32["jacobi"] * 1e-3) / 1e9,
                           "fp32_residual_ms": k32["residual"], "fp64_jacobi_ms": k64f["jacobi"],
                           "fp64_jacobi_gbs": gbs_jac64, "fcg_spmv_dots_ms": k64f["fcg_spmv_dots"],
                           # pw = A pv (row kernel) then the three dots (r, pw, oq against pv)
                           "fcg_spmv_dots_gbs": ((ib64 + vb64) * nnz + rb64 + 4 * (n + 1) + 48 * n) / (k64f["fcg_spmv_dots"] * 1e-3) / 1e9,
                           "fp32_jacobi_fp64_out_ms": k32["jacobi_fp64_out"],
                           "fcg_update_ms": k32["fcg_update"],
                           "fcg_update_gbs": 80 * n / (k32["fcg_update"] * 1e-3) / 1e9},
        "kernels_coarse_levels_fp32_jacobi_ms": [round(k["jacobi"], 4) for k in lvl],
        "vcycle": vcycle_roofline(vc_ms, inf32, params("FP32"), peak, peak_kind),
        "roofline": {"kernel": (("k_rowop_slpat<OP_JACOBI,float>" if (form0 == "sliced" and ib32 == 0) else
                                 kname0 + ("OP_JACOBI,Coded<float>>" if vb32 == 1 else "OP_JACOBI,float>"))
                                + " (FP32 l1-Jacobi sweep, level 0)"),
                     "format": ("pattern-indexed rows (1 byte per row)" if ib32 == 0 else f"int{8 * ib32} columns")
                               + ", " + ("1-byte value codes" if vb32 == 1 else "FP32 values"),
                     "bound": "hbm", "achieved": gbs_jac32, "peak": peak, "unit": "GB/s",
                     "frac": gbs_jac32 / peak, "peak_kind": f"{peak_kind} hbm_gbs (copy)",
                     "bytes_per_launch": bytes_jac32,
                     "traffic": (int(TRAFFIC_RATIO[(ib32, vb32, form0)] * bytes_jac32)
                                 if a.workload.startswith("poisson27") and (ib32, vb32, form0) in TRAFFIC_RATIO
                                 else None)},
        "cold_first_call": dict(cold, what="the first set-up + solve of each form in the process (threads-per-row "
                                "autotuner running, kernels loading); the timed steps reuse the tuned choices"),
        "gpu_launches": int(round(launches32)),
        "e2e": {"value": e2e_ms / 1e3, "unit": "s", "h2d_bytes_per_step": int(row.nbytes + col.nbytes + val.nbytes + b.nbytes),
                "d2h_bytes_per_step": int(n * 8), "path": "bcmgx_setup(host CSR) + bcmgx_solve(host b, x), pinned"},
    }
    if clk:
        line["clocks"] = clk
    return line, {"x32": x32, "x64": x64}


# DRAM bytes (read + write) of one level-0 FP32 Jacobi launch as a multiple of its algorithmic
# bytes, per (index bytes, value bytes, kernel form): measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum of single launches) on the 27-point 100^3 case: the plain kernel with int32
# columns and with int16 offsets, the staged kernel with int16 offsets (FP32 values, and one-byte
# value codes), the sliced kernel with int16 offsets and codes (its padding included, its row
# offsets not read), the pattern-indexed sliced kernel (index bytes 0: its padding codes read, the
# row offsets counted in the algorithmic bytes not read, part of x served by L2); scaled by the
# algorithmic bytes to the other 27-point workloads.
TRAFFIC_RATIO = {(4, 4, "plain"): 0.99983, (2, 4, "plain"): 1.00115, (2, 4, "staged"): 1.01173,
                 (2, 1, "staged"): 0.99886, (2, 1, "sliced"): 0.99216, (0, 1, "sliced"): 0.88800}


def _spmv(row, col, val, x):
    import scipy.sparse as sp
    n = row.size - 1
    return sp.csr_matrix((val, col, row), shape=(n, n)) @ x


def run_adjoint(a, rank=0, world=1, local_rank=0, steps=None, warmup=None):
    """Differentiated solve (7-point FV diffusion 96^3, kappa = exp(theta)): forward FCG+BCMG to
    1e-10, backward = adjoint solve on the same hierarchy, chained to dL/dtheta by torch; the
    gradient is checked along random directions against FP64 central differences and against
    the gradient of a fresh plain-FP64 solve. At N > 1 every rank runs its own replica and the
    time is the slowest rank's."""
    import torch
    import bootcmatchgx_b200 as bx
    from bootcmatchgx_b200 import autograd, problems
    dev = torch.device("cuda", local_rank)
    steps = a.steps if steps is None else steps
    warmup = a.warmup if warmup is None else warmup
    cfg = ADJOINT
    g = cfg["grid"]
    n = g[0] * g[1] * g[2]
    theta0 = torch.from_numpy(problems.gaussian_random_field(g, 8.0, 2.0, cfg["theta_seed"]).reshape(-1, order="F")).to(dev)
    asm = problems.DiffusionAssembler(*g, dev)
    rng = np.random.default_rng(cfg["noise_seed"])
    b = torch.ones(n, dtype=torch.float64, device=dev)
    prm = autograd.default_params(rtol=cfg["rtol"], vcycle_precision="FP32")
    prm64 = autograd.default_params(rtol=cfg["rtol"], vcycle_precision="FP64")
    with torch.no_grad():
        x_obs = autograd.solve(asm.row, asm.col, asm.values(torch.exp(theta0)), b, prm64)
        x_obs = x_obs + 1e-3 * torch.from_numpy(rng.standard_normal(n)).to(dev)
    theta = (theta0 + 0.1 * torch.from_numpy(rng.standard_normal(n)).to(dev)).detach()

    def fwd_bwd(p):
        th = theta.clone().requires_grad_(True)
        x = autograd.solve(asm.row, asm.col, asm.values(torch.exp(th)), b, p)
        L = 0.5 * ((x - x_obs) ** 2).sum()
        (gr,) = torch.autograd.grad(L, th)
        return L.detach(), gr

    def xsol(th, p):
        with torch.no_grad():
            return autograd.solve(asm.row, asm.col, asm.values(torch.exp(th)), b, p)

    for _ in range(max(1, warmup)):
        fwd_bwd(prm)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        L, grad = fwd_bwd(prm)
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / steps, world, dev)
    _, grad64 = fwd_bwd(prm64)
    tight = autograd.default_params(rtol=1e-13, vcycle_precision="FP64")
    _, grad_t = fwd_bwd(tight)
    errs, errs_t = [], []
    h = cfg["step"]
    for _ in range(cfg["directions"]):
        d = torch.from_numpy(rng.standard_normal(n)).to(dev)   # N(0, I) direction, per-cell step h
        # L(theta + h d) - L(theta - h d) as one sum of per-cell differences,
        # 0.5 (x+ - x-) . (x+ + x- - 2 x_obs): the same number as the difference of the two losses
        # (each about 1.4e5) without the cancellation of their last digits
        xp, xm = xsol(theta + h * d, tight), xsol(theta - h * d, tight)
        fd = 0.5 * ((xp - xm) * (xp + xm - 2.0 * x_obs)).sum() / (2 * h)
        errs.append(abs(float(fd - (grad * d).sum())) / abs(float(fd)))
        errs_t.append(abs(float(fd - (grad_t * d).sum())) / abs(float(fd)))
    return {"metric": "differentiated solve: forward+backward s (FP32 V-cycle)", "value": ms / 1e3, "unit": "s",
            "higher_is_better": False, "workload": "diffusion7_96_adjoint", "rows": n, "nnz": int(asm.nnz),
            "n_gpus": world, "steps": steps, "warmup": warmup,
            "config": {"problem": "7-point FV diffusion 96^3, kappa = exp(theta), theta GRF (length 8, sigma 2, seed 5); "
                                  "x_obs = x(theta0) + N(0,1e-3); theta = theta0 + 0.1 N(0,1); L = 0.5||x - x_obs||^2",
                       "rtol": cfg["rtol"], "fd_step": h, "directions": cfg["directions"]},
            "fd": "central differences of L on FP64 solves to rtol 1e-13 (the loss difference summed per cell), "
                  "directions d ~ N(0, I)",
            "grad_rel_err_vs_central_fd_max": max(errs), "grad_rel_err_vs_central_fd_median": float(np.median(errs)),
            "grad_fp64_rel_err_vs_central_fd_max": max(errs_t),
            "grad_rel_err_vs_fresh_fp64": float((grad - grad64).norm() / grad64.norm()), "loss": float(L)}


def run_batch(a, rank=0, world=1, local_rank=0, steps=None, warmup=None):
    """256 independent 7-point Poisson systems, box sides uniform in 10..46 (seed 4), diagonal shift
    uniform[0, 0.5], FP32 V-cycle, rhs uniform[-1,1]: one CUDA-graph launch for all solves (the
    lockstep form; the per-system-branch form beside it) vs a sequential loop of single solves
    (same hierarchies, warm graphs). At N > 1 rank r takes
    systems r, r + N, ... (bootcmatchgx_b200.replicas) on its own GPU, with no communication; the
    time is the slowest rank's and the value counts all 256 systems."""
    import scipy.sparse as sp
    import torch
    import bootcmatchgx_b200 as bx
    from bootcmatchgx_b200 import replicas
    dev = torch.device("cuda", local_rank)
    steps = a.steps if steps is None else steps
    warmup = a.warmup if warmup is None else warmup
    rng = np.random.default_rng(4)
    systems, rhs, rows = [], [], 0
    for _ in range(256):
        dims = [int(d) for d in rng.integers(10, 47, size=3)]
        shift = rng.uniform(0.0, 0.5)
        r, c, v = bx.laplacian_3d(7, *dims)
        v = v + shift * (c == np.repeat(np.arange(r.size - 1), np.diff(r)))
        systems.append((r, c, v))
        rows += r.size - 1
    for r, _, _ in systems:
        rhs.append(rng.uniform(-1, 1, r.size - 1))
    mine = replicas.systems_of_rank(len(systems), rank, world)
    sysm = [systems[k] for k in mine]
    bs = [torch.from_numpy(rhs[k]).to(dev) for k in mine]
    p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=1e-8, dispnorm=0, vcycle_precision="FP32")
    nthreads = min(16, os.cpu_count() or 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    B = bx.Batch(sysm, p, nthreads=nthreads)
    torch.cuda.synchronize()
    t_setup = max_over_ranks(time.perf_counter() - t0, world, dev)
    t0 = time.perf_counter()
    xs, infos = B.solve(bs)   # sets up the lockstep groups (the systems' block-diagonal unions) and the graph
    torch.cuda.synchronize()
    t_first = max_over_ranks(time.perf_counter() - t0, world, dev)
    for _ in range(max(0, warmup - 1)):
        B.solve(bs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        xs, infos = B.solve(bs)
    torch.cuda.synchronize()
    t_batch = max_over_ranks((time.perf_counter() - t0) / steps, world, dev)
    # the per-system form of the same batch (one graph branch per system) for comparison
    B.set_lockstep(False)
    for _ in range(max(1, warmup)):
        B.solve(bs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        B.solve(bs)
    torch.cuda.synchronize()
    t_branch = max_over_ranks((time.perf_counter() - t0) / steps, world, dev)
    B.set_lockstep(True)
    hs = [B.hierarchy(k) for k in range(len(sysm))]
    for k, h in enumerate(hs):   # warm each single-solve graph
        h.solve(bs[k])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        for k, h in enumerate(hs):
            h.solve(bs[k])
    torch.cuda.synchronize()
    t_seq = max_over_ranks((time.perf_counter() - t0) / steps, world, dev)
    worst = 0.0
    for k, (r, c, v) in enumerate(sysm):
        A = sp.csr_matrix((v, c, r), shape=(r.size - 1,) * 2)
        bb = bs[k].cpu().numpy()
        worst = max(worst, float(np.linalg.norm(bb - A @ xs[k].cpu().numpy()) / np.linalg.norm(bb)))
    worst = max_over_ranks(worst, world, dev)
    it_lo = -max_over_ranks(-min(i["niter"] for i in infos), world, dev)
    it_hi = max_over_ranks(max(i["niter"] for i in infos), world, dev)
    B.free()
    return {"metric": "batched solves/s (256 uneven 7-point systems, one graph launch)", "value": 256 / t_batch,
            "unit": "solves/s", "higher_is_better": True, "workload": "batch256_poisson7", "n_gpus": world,
            "form": "lockstep: every step one kernel over the systems of a group (groups of at most 32 systems "
                    "with the same level count, neighbouring sizes), one graph for all groups",
            "sequential_solves_per_s": 256 / t_seq, "speedup_vs_sequential": t_seq / t_batch,
            "per_system_graph_solves_per_s": 256 / t_branch,
            "batch_solve_ms": t_batch * 1e3, "sequential_ms": t_seq * 1e3, "setup_ms": t_setup * 1e3,
            "first_solve_ms": t_first * 1e3,
            "total_rows": rows, "iters_min_max": [int(it_lo), int(it_hi)],
            "max_rel_residual": worst, "steps": steps, "warmup": warmup,
            "config": {"systems": 256, "sides": "uniform 10..46 (numpy default_rng(4))", "shift": "uniform[0,0.5]",
                       "vcycle": "fp32", "rtol": 1e-8, "setup_threads": nthreads,
                       "parallelism": f"systems round robin over {world} GPU(s), one batch graph per GPU"}}


def block_kernel_rooflines(t, n, nnz, k):
    """Level-0 block kernels of the FP32-cycle multi-RHS solve (bcmgx_time_block_kernels, CUDA
    events, zero inputs): ms per launch and HBM GB/s of the algorithmic bytes (matrix once, every
    block read or written once: the gathers of X from L1/L2 are not counted) against the measured
    copy peak. The FP32 sweep reads the FP32 matrix values (8 bytes per entry with the int32
    column), the FP64 kernels 12 bytes per entry."""
    peak, kind = read_peaks()
    blk4, blk8 = 4.0 * n * k, 8.0 * n * k
    alg = {"jacobi": 8 * nnz + 4 * (n + 1) + 4 * n + 3 * blk4,
           "residual": 8 * nnz + 4 * (n + 1) + 3 * blk4,
           "spmm": 12 * nnz + 4 * (n + 1) + 2 * blk8,
           "fcg_spmm_dots": 12 * nnz + 4 * (n + 1) + 4 * blk8}
    out = {"peak_gbs": peak, "peak_kind": kind}
    for key, b in alg.items():
        ms = t[key]
        out[key] = {"ms": ms, "algorithmic_bytes": int(b), "gbs": b / ms / 1e6, "frac": b / ms / 1e6 / peak}
    return out


def run_multi(a, rank=0, world=1, local_rank=0, steps=None, warmup=None, kernels=True):
    """The 27-point 100^3 Poisson matrix with 32 right-hand sides (uniform[-1,1], numpy
    default_rng(6)) solved to 1e-8 in one block solve (CSR SpMM throughout, FP32 V-cycle) vs a
    sequential loop of 32 single solves on the same hierarchy; also the block FP64-cycle solve,
    the level-0 block kernels (CUDA events, HBM GB/s of their algorithmic bytes) and the public
    SpMM call. At N > 1 rank r solves a contiguous slice of the 32 columns
    (bootcmatchgx_b200.replicas) with its own hierarchy on its own GPU, with no communication;
    times are the slowest rank's and the value counts all 32 columns."""
    import scipy.sparse as sp
    import torch
    import bootcmatchgx_b200 as bx
    from bootcmatchgx_b200 import replicas
    dev = torch.device("cuda", local_rank)
    steps = a.steps if steps is None else steps
    warmup = a.warmup if warmup is None else warmup
    ktot = 32
    row, col, val = bx.laplacian_3d(27, 100, 100, 100)
    n, nnz = row.size - 1, col.size
    Ball = np.random.default_rng(6).uniform(-1.0, 1.0, (n, ktot))
    cols = replicas.columns_of_rank(ktot, rank, world)
    k = len(cols)
    B = np.ascontiguousarray(Ball[:, cols.start:cols.stop])
    d = [torch.from_numpy(x_).to(dev) for x_ in (row, col, val)]
    Bd = torch.from_numpy(B).to(dev)
    X = torch.zeros_like(Bd)
    A = sp.csr_matrix((val, col, row), shape=(n, n))
    out = {}
    for prec in ("FP32", "FP64"):
        p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=1e-8, dispnorm=0, vcycle_precision=prec)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h = bx.Hierarchy(d[0], d[1], d[2], p)
        torch.cuda.synchronize()
        t_setup = max_over_ranks(time.perf_counter() - t0, world, dev)
        for _ in range(max(1, warmup)):
            X.zero_()
            h.solve_multi(Bd, X)
        ts = []
        for _ in range(steps):
            X.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, infos = h.solve_multi(Bd, X)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        t_block = max_over_ranks(float(np.median(ts)), world, dev)
        Xh = X.cpu().numpy()
        rel = np.linalg.norm(B - A @ Xh, axis=0) / np.linalg.norm(B, axis=0)
        res = {"block_ms": t_block * 1e3, "solves_per_s": ktot / t_block, "setup_ms": t_setup * 1e3,
               "iters_min_max": [int(-max_over_ranks(-min(i["niter"] for i in infos), world, dev)),
                                 int(max_over_ranks(max(i["niter"] for i in infos), world, dev))],
               "max_rel_residual": max_over_ranks(float(rel.max()), world, dev)}
        if prec == "FP32":
            xs = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(k)]
            colv = [Bd[:, j].contiguous() for j in range(k)]
            h.solve(colv[0], xs[0])   # builds the single-solve graph
            ts = []
            for _ in range(max(1, steps // 2)):
                for x_ in xs:
                    x_.zero_()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                for j in range(k):
                    h.solve(colv[j], xs[j])
                torch.cuda.synchronize()
                ts.append(time.perf_counter() - t0)
            t_seq = max_over_ranks(float(np.median(ts)), world, dev)
            res["sequential_ms"] = t_seq * 1e3
            res["sequential_solves_per_s"] = ktot / t_seq
            res["speedup_vs_sequential"] = t_seq / t_block
            res["max_rel_diff_vs_single"] = max_over_ranks(
                max(float(torch.linalg.norm(X[:, j] - xs[j]) / torch.linalg.norm(xs[j])) for j in range(k)), world, dev)
            if kernels:
                res["kernels_level0"] = block_kernel_rooflines(h.time_block_kernels(k, reps=20), n, nnz, k)
        h.free()
        out[prec] = res
    f32 = out["FP32"]
    line = {"metric": "multi-RHS solves/s (27-point 100^3, 32 right-hand sides, one block solve)",
            "value": f32["solves_per_s"], "unit": "solves/s", "higher_is_better": True, "workload": "poisson27_100_x32",
            "n_gpus": world, "fp32": f32, "fp64": out["FP64"], "steps": steps, "warmup": warmup,
            "config": {"rows": n, "nnz": nnz, "rhs": ktot, "rhs_dist": "uniform[-1,1] (numpy default_rng(6))",
                       "rtol": 1e-8, "x0": 0,
                       "parallelism": f"columns in contiguous slices over {world} GPU(s), one hierarchy per GPU"}}
    if kernels and world == 1:
        # the public SpMM call Y = A X for the 32-column block: CSR validation on the device, a host
        # round trip for its verdict, then the kernel (the kernel alone: fp32.kernels_level0.spmm)
        Y = torch.empty_like(Bd)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(3):
            bx.spmm(d[0], d[1], d[2], Bd, Y)
        reps = 20
        e0.record()
        for _ in range(reps):
            bx.spmm(d[0], d[1], d[2], Bd, Y)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        alg = nnz * 12 + (n + 1) * 4 + 2 * n * k * 8
        peak, peak_kind = read_peaks()
        line["spmm_call"] = {"ms": ms, "what": "bcmgx_spmm: validation + host round trip + kernel",
                             "algorithmic_bytes": alg, "gbs": alg / ms / 1e6, "peak_gbs": peak,
                             "frac": alg / ms / 1e6 / peak, "peak_kind": peak_kind}
    return line


def profile_multi_step(a):
    """W warm-up block solves, then exactly one (27-point 100^3, 32 right-hand sides, FP32 V-cycle,
    stream-driven so that every kernel is a separate launch); prints the launch counts."""
    import torch
    import bootcmatchgx_b200 as bx
    dev = torch.device("cuda", 0)
    row, col, val = bx.laplacian_3d(27, 100, 100, 100)
    d = [torch.from_numpy(x_).to(dev) for x_ in (row, col, val)]
    Bd = torch.from_numpy(np.random.default_rng(6).uniform(-1.0, 1.0, (row.size - 1, 32))).to(dev)
    X = torch.zeros_like(Bd)
    p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=1e-8, dispnorm=0, vcycle_precision="FP32",
                          use_graph=0)
    h = bx.Hierarchy(d[0], d[1], d[2], p)
    L = bx.lib()
    c0 = L.bcmgx_launch_count()
    for _ in range(a.warmup):
        X.zero_()
        h.solve_multi(Bd, X)
    c1 = L.bcmgx_launch_count()
    X.zero_()
    _, infos = h.solve_multi(Bd, X)
    torch.cuda.synchronize()
    c2 = L.bcmgx_launch_count()
    h.free()
    print(json.dumps({"warmup_launches": c1 - c0, "launches_before_step": c1, "step_launches": c2 - c1,
                      "niter_max": max(i["niter"] for i in infos)}), flush=True)


def profile_step(a, wl):
    """W warm-up steps, then exactly one set-up + solve (FP32 V-cycle) on device-resident data;
    prints how many library kernels the warm-up and the step launched. The solve is
    stream-driven (use_graph = 0: the same kernels as the captured solve, launched one by one),
    so that a profiler sees every kernel of the step."""
    import torch
    import bootcmatchgx_b200 as bx
    dev = torch.device("cuda", 0)
    row, col, val, xs, b = build_problem(wl)
    d = [torch.from_numpy(x_).to(dev) for x_ in (row, col, val, b)]
    x = torch.zeros(row.size - 1, dtype=torch.float64, device=dev)
    p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=RTOL, dispnorm=0, vcycle_precision="FP32",
                          use_graph=0)
    L = bx.lib()
    c0 = L.bcmgx_launch_count()
    for _ in range(a.warmup):
        h = bx.Hierarchy(d[0], d[1], d[2], p)
        x.zero_()
        h.solve(d[3], x)
        h.free()
    c1 = L.bcmgx_launch_count()
    h = bx.Hierarchy(d[0], d[1], d[2], p)
    x.zero_()
    _, info = h.solve(d[3], x)
    h.free()
    torch.cuda.synchronize()
    c2 = L.bcmgx_launch_count()
    print(json.dumps({"warmup_launches": c1 - c0, "step_launches": c2 - c1, "niter": info["niter"]}), flush=True)


def run_dist(a, wl, rank=0, world=1, local_rank=0, parts=2):
    """The row-partitioned path (the reference's multi-rank solve): set-up + FCG solve to 1e-8 with
    the FP64 V-cycle, rows split into equal blocks. With one process (world 1) all `parts` blocks
    run on one GPU (the local form: exchanges as device copies); under torchrun every rank holds
    one block on its own GPU and exchanges over NCCL (the communicator made from a unique id that
    rank 0 shares through torch.distributed). Times: CUDA events, the slowest rank's."""
    import torch
    import bootcmatchgx_b200 as bx
    dev = torch.device("cuda", local_rank)
    row, col, val, xs, b = build_problem(wl)
    n = row.size - 1
    nparts = world if world > 1 else parts
    offs = [n * k // nparts for k in range(nparts + 1)]
    p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=RTOL, dispnorm=0, vcycle_precision="FP64")
    comm = None
    if world > 1:
        import torch.distributed as dist
        uid = [bx.nccl_unique_id() if rank == 0 else None]
        dist.broadcast_object_list(uid, src=0)
        comm = bx.nccl_comm(world, rank, uid[0])
        r0, r1 = offs[rank], offs[rank + 1]
        e0_, e1_ = row[r0], row[r1]
        d = [torch.from_numpy(np.ascontiguousarray(row[r0:r1 + 1] - e0_)).to(dev),
             torch.from_numpy(np.ascontiguousarray(col[e0_:e1_])).to(dev),
             torch.from_numpy(np.ascontiguousarray(val[e0_:e1_])).to(dev)]
        bd = torch.from_numpy(np.ascontiguousarray(b[r0:r1])).to(dev)
    else:
        d = [torch.from_numpy(x_).to(dev) for x_ in (row, col, val)]
        bd = torch.from_numpy(b).to(dev)
    x = torch.zeros_like(bd)

    def step():
        D = (bx.Dist.nccl(d[0], d[1], d[2], offs[rank], n, comm, world, p) if world > 1
             else bx.Dist.local(d[0], d[1], d[2], offs, p))
        x.zero_()
        _, info = D.solve(bd, x)
        inf = D.info()
        D.free()
        return info, inf
    try:
        for _ in range(max(1, a.warmup)):
            step()
        torch.cuda.synchronize()
        steps = max(1, min(a.steps, 5))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = [step() for _ in range(steps)]
        e1.record()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps, world, dev)
        xh = x.cpu().numpy()
        err = None
        if xs is not None:
            xs_mine = xs[offs[rank]:offs[rank + 1]] if world > 1 else xs
            err = max_over_ranks(float(np.linalg.norm(xh - xs_mine) / np.linalg.norm(xs_mine)), world, dev)
    finally:
        if comm is not None:
            bx.nccl_comm_destroy(comm)
    info, inf = res[-1]
    return {"metric": "row-partitioned set-up + solve s to rel-res 1e-8 (FP64 V-cycle)", "value": ms / 1e3,
            "unit": "s", "higher_is_better": False, "workload": a.workload, "n_gpus": world, "ranks": nparts,
            "transport": "nccl (one block per GPU)" if world > 1 else "local (all blocks on one GPU, device copies)",
            "setup_ms": float(np.mean([r[1]["setup_ms"] for r in res])),
            "solve_ms": float(np.mean([r[0]["solve_ms"] for r in res])), "niter": info["niter"],
            "levels": inf["n"], "level_nnz": inf["nnz"], "err_vs_xstar": err, "steps": steps,
            "config": {"rows": int(n), "nnz": int(col.size), "blocks": "equal consecutive row blocks", "rtol": RTOL}}


def run_small(a, name, rank=0, world=1, local_rank=0, steps=10, warmup=3):
    """A small workload (the 7-point 50^3 Poisson system by default: 125,000 rows, L2-resident)
    through the same step as the headline: set-up + FCG solve to 1e-8, FP32 and FP64 V-cycles,
    CUDA events, the slowest rank's time; rank 0 also compares the level sizes and iterations
    with the oracle's (a fraction of a second on the host at this size)."""
    import torch
    import bootcmatchgx_b200 as bx
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)
    wl = WORKLOADS[name]
    row, col, val, xs, b = build_problem(wl)
    d = [torch.from_numpy(x_).to(dev) for x_ in (row, col, val, b)]
    x = torch.zeros(row.size - 1, dtype=torch.float64, device=dev)
    out = {"workload": name, "rows": int(row.size - 1), "nnz": int(col.size), "steps": steps, "warmup": warmup,
           "n_gpus": world}
    for prec in ("FP32", "FP64"):
        p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=RTOL, dispnorm=0, vcycle_precision=prec,
                              stream=stream.cuda_stream)

        def step():
            h = bx.Hierarchy(d[0], d[1], d[2], p)
            x.zero_()
            _, info = h.solve(d[3], x)
            inf = h.info()
            h.free()
            return info, inf
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = [step() for _ in range(steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps, world, dev)
        xh = x.cpu().numpy()
        out[prec.lower()] = {"ms_per_step": ms, "setup_ms": float(np.mean([r[1]["setup_ms"] for r in res])),
                             "solve_ms": float(np.mean([r[0]["solve_ms"] for r in res])), "niter": res[-1][0]["niter"],
                             "err_vs_xstar": None if xs is None else float(np.linalg.norm(xh - xs) / np.linalg.norm(xs)),
                             "levels": res[-1][1]["n"], "level_nnz": res[-1][1]["nnz"]}
    if rank == 0:
        from oracle import pyoracle as O
        O.num_threads(host_info()["cpus_available"])
        ts, tv, xo, io, lv = oracle_solve(O, O.Matrix.from_csr(row, col, val), b)
        gl = list(zip(out["fp64"]["levels"], out["fp64"]["level_nnz"]))
        out["parity"] = {"levels_equal": gl == [tuple(t) for t in lv], "niter_oracle": io["niter"],
                         "niter_fp64": out["fp64"]["niter"], "oracle_s": ts + tv}
    return out


def secondary_configs(a, rank, world, local_rank):
    """The other configurations, each in a bounded number of steps, as extra keys of the headline
    line (every rank runs them in the same order, so that their max-over-ranks reductions pair
    up): C1 (7-point 50^3), C5 (differentiated 96^3 diffusion), C4a (256 uneven systems in one
    graph launch) and C4b (32 right-hand sides)."""
    jobs = [("poisson7_50", lambda: run_small(a, "poisson7_50", rank, world, local_rank)),
            ("adjoint_diffusion7_96", lambda: run_adjoint(a, rank, world, local_rank, steps=3, warmup=1)),
            ("batch256_poisson7", lambda: run_batch(a, rank, world, local_rank, steps=3, warmup=2)),
            ("poisson27_100_x32", lambda: run_multi(a, rank, world, local_rank, steps=3, warmup=1, kernels=False))]
    if world == 1:
        # the row-partitioned path on the headline workload, two row blocks on this GPU
        short = argparse.Namespace(**dict(vars(a), steps=2, warmup=1))
        jobs.append(("partitioned_2blocks_" + a.workload,
                     lambda: run_dist(short, WORKLOADS[a.workload], 0, 1, local_rank, parts=2)))
    out = {}
    for name, fn in jobs:
        t0 = time.perf_counter()
        try:
            out[name] = fn()
        except Exception as e:   # reported in the line; the headline stands
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["wall_s"] = time.perf_counter() - t0
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="poisson27_160", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true", help="leave out the other configurations' summaries")
    ap.add_argument("--adjoint", action="store_true", help="run the differentiated-solve configuration instead")
    ap.add_argument("--batch", action="store_true", help="run the batched-systems configuration instead")
    ap.add_argument("--multi", action="store_true", help="run the 32-right-hand-side configuration instead")
    ap.add_argument("--dist", type=int, default=0, metavar="P",
                    help="run the row-partitioned path instead: P blocks on one GPU, or one block per rank under "
                         "torchrun (P is then the world size)")
    ap.add_argument("--cpu-leg", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--profile-step", action="store_true",
                    help="only W warm-up steps and one FP32 step (for ncu launch lists); prints the launch counts")
    a = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    wl = WORKLOADS[a.workload]
    if a.cpu_leg:   # the CPU baseline's child process (cpu_baseline)
        line, ora = cpu_baseline_leg(wl, runs=a.steps)
        np.savez(a.cpu_leg, line=json.dumps(line), x=ora["x"], niter=ora["niter"], levels=np.array(ora["levels"]))
        return
    if a.impl == "reference":
        line = reference_arm(a, wl, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if a.profile_step:
        if a.multi:
            profile_multi_step(a)
        else:
            profile_step(a, wl)
        return
    import torch
    torch.cuda.set_device(local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        line = None
        if a.adjoint:
            line = run_adjoint(a, rank, world, local_rank)
        elif a.batch:
            line = run_batch(a, rank, world, local_rank)
        elif a.multi:
            line = run_multi(a, rank, world, local_rank)
        elif a.dist:
            line = run_dist(a, wl, rank, world, local_rank, parts=a.dist)
        else:
            line, extra = run_ours(a, wl, rank, world, local_rank)
            if not a.no_secondary:
                sec = secondary_configs(a, rank, world, local_rank)
                if line is not None:
                    line["secondary"] = sec
            if rank == 0 and world == 1 and not a.no_cpu_baseline:
                cb, ora = cpu_baseline(a.workload)
                line["cpu_baseline"] = cb
                x64 = extra["x64"]
                gl = list(zip(line["breakdown"]["levels"], line["breakdown"]["level_nnz"]))
                line["parity"] = {
                    "levels_equal": gl == [tuple(t) for t in ora["levels"]],
                    "level_sizes_oracle": ora["levels"], "niter_oracle": ora["niter"],
                    "niter_fp64": line["fp64"]["niter"], "niter_fp32": line["breakdown"]["niter"],
                    "fp64_rel_diff_vs_oracle_solution": float(np.linalg.norm(x64 - ora["x"]) / np.linalg.norm(ora["x"])),
                    "fp32_rel_diff_vs_oracle_solution": float(np.linalg.norm(extra["x32"] - ora["x"]) / np.linalg.norm(ora["x"])),
                    "what": "GPU hierarchy sizes, iterations and solutions against the oracle's run on the same inputs"}
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
