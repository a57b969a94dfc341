#!/usr/bin/env python
"""Factor + solve benchmark of the FPLUS path on B200 (one JSON line on stdout, rank 0).

Workload (default ``pencil``): the shift-invert pencil A - sigma B, complex128, 8 Fourier modes x 4 fields x 1024
Chebyshev modes (n = 32,768), banded blocks of half-bandwidth 6, 8 dense tau rows and 8 dense tau columns over all n,
magnitudes log-uniform in [1e-6, 1e6] with seeded phases, sigma = 0.3 + 1.7i; b ~ N(0, 1) complex, nrhs 1.  ``--workload
convdiff2d`` runs the 100 x 100 convection-diffusion stencil (n = 10,000, real) instead.  Synthetic, seeded.

One step = fplus_factor (permutation, Ruiz, the multifrontal LU) + fplus_solve on one matrix, the symbolic analysis
(fplus_analyze_opts: done once per pattern, reported as analyze_ms) reused across steps.  The metric is milliseconds
per step with the solution at backward error <= 1e-14 (checked after the timed steps; lower is better).

* value -- device-timed (CUDA events on the stream the library runs on) with the matrix and right-hand side resident in
  HBM (fplus_b200_factor_dev / fplus_b200_solve_dev); L2 flushed (a 512 MiB write) between steps, outside the events.
* e2e   -- the same step through the public fplus_factor / fplus_solve with pinned host buffers: the host-to-device copy
  of the values and the right-hand side and the device-to-host copy of the solution are inside the timed region.
* roofline -- the dominant kernel class of the factorization, from a separate step with the library's per-class CUDA
  event timing on: achieved algorithmic rate / measured peak.
* cpu_baseline -- the reference's own CPU build (oracle/_ref/libfplusref.so: the FPLUS sources, OpenMP + OpenBLAS, all
  host threads) timed on a bounded sample of the same generator (1 Fourier mode, n = 4096), reported as measured.
* c1_pair -- the 100 x 100 stencil (the reference's CPU-runnable configuration) in full on both sides: this library's
  device and end-to-end times, the reference at all host threads and at 1 thread.
* --impl reference -- the reference's CPU build on this arm's configuration, with the static orders of
  tests/golden/orders.npz (libfplus.so is not loaded).  The stencil runs in full; for the pencil the arm prints the
  unavailable line with the reference's measured times on the same generator at 1 and 2 Fourier modes.

Multi-GPU: one factorization does not shard; N ranks run N independent replicas ("replicas only"); the line reports
the slowest rank's ms per step divided by N (the job's ms per factorization) with scaling "weak".
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def workload(name, modes=8):
    from fplus_b200 import workloads as W
    if name == "pencil":
        n, Ap, Ai, Ax = W.pencil(modes=modes)
        desc = {"workload": f"pencil A - sigma B, {modes} Fourier x 4 fields x 1024 Chebyshev (n={n}), complex128, "
                            "half-bandwidth 6, 8 dense tau rows + 8 dense tau columns, |a| log-uniform [1e-6, 1e6], "
                            "sigma=0.3+1.7i", "n": n, "nnz": int(Ap[-1]), "nrhs": 1}
    elif name == "convdiff2d":
        n, Ap, Ai, Ax = W.convdiff2d(100, 1)
        desc = {"workload": "2D convection-diffusion 5-point, 100x100 grid (n=10000), float64", "n": n,
                "nnz": int(Ap[-1]), "nrhs": 1}
    else:
        raise SystemExit(f"unknown workload {name}")
    b = W.rhs(n, 1, np.iscomplexobj(Ax), 2)[0]
    return n, Ap, Ai, Ax, b, desc


def load_orders(name, Ap, Ai):
    """The committed static orders of a workload (tests/golden/orders.npz, written by tests/golden/make_orders.py from
    this library's analysis): the reference's arm injects them into the reference's own fplus_analyze without loading
    libfplus.so.  (row_perm, col_perm, dense-row mask, dense-column mask)."""
    z = np.load(os.path.join(ROOT, "tests", "golden", "orders.npz"))
    chk = np.array([int(Ap[-1]), int(np.sum(Ap, dtype=np.int64)), int(np.sum(Ai * (np.arange(Ai.size) % 7 + 1), dtype=np.int64))])
    if not np.array_equal(chk, z[name + "__pattern"]):
        raise SystemExit(f"orders.npz: the pattern of {name} has changed (rerun tests/golden/make_orders.py)")
    return z[name + "__row_perm"], z[name + "__col_perm"], z[name + "__trow"], z[name + "__tcol"]


def reference_time(name, gen, reps):
    """The reference's CPU build (oracle/_ref/libfplusref.so: the FPLUS sources, OpenMP + OpenBLAS) on one workload,
    factor + solve per step (its analysis done once, outside the timing, on the committed orders): (median ms, berr,
    n).  Threads: OMP_NUM_THREADS / OPENBLAS_NUM_THREADS as set by the caller, else all host cores."""
    import oracle as O
    from fplus_b200 import workloads as W
    n, Ap, Ai, Ax = gen()
    rp, cp, trow, tcol = load_orders(name, Ap, Ai)
    b = W.rhs(n, 1, np.iscomplexobj(Ax), 2)[0]
    R = O.RefLU(n, Ap, Ai, None, cp, trow, tcol, postorder=0)        # the injected order, no postorder: cp as given
    assert np.array_equal(R.row_perm, rp) and np.array_equal(R.col_perm, cp)
    times, be = [], None
    for _ in range(reps):
        t0 = time.perf_counter()
        R.refactor(Ax)
        x = R.solve(b)
        times.append((time.perf_counter() - t0) * 1e3)
        be = O.backward_error(n, Ap, Ai, Ax, x, b)
    del R
    return float(np.median(times)), be, n


def ref_threads():
    t = os.environ.get("OMP_NUM_THREADS")
    return int(t) if t and t.isdigit() else os.cpu_count()


# ------------------------------------------------------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"fplus_b200_clocks_{os.getpid()}_{gpu_index}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1])); smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------------------------------- peaks
def fp64_peak_tflops(torch, cplx):
    """cuBLAS FP64 GEMM throughput on this GPU (the roofline of an FP64 tensor-core kernel: the driver's measured peaks
    file covers bf16 and HBM only): complex128 (ZGEMM, 8 flops per multiply-add) or float64, 8192^3, best of 5."""
    dt = torch.complex128 if cplx else torch.float64
    m = 8192
    a = torch.randn(m, m, dtype=dt, device="cuda")
    b = torch.randn(m, m, dtype=dt, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(); torch.matmul(a, b); e1.record(); torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return (8.0 if cplx else 2.0) * m ** 3 / (best * 1e-3) / 1e12


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# ------------------------------------------------------------------------------------------------------------- ranks
def allreduce_max(value: float, device) -> float:
    """The maximum of a per-rank value over all ranks (every rank gets it); the value itself with one rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------------------------------------------------- arms
def run_profile_once(args):
    """One factorization and solve inside a profiler range (after a warm factorization and solve that size every buffer),
    then the per-class algorithmic flops and bytes of that factorization (the library's own counts) as one JSON line.
    --profile-workload: the benchmark workload (--workload), the 3D stencil (stencil3d, --precision-grid), or the
    17-decade random configuration (random, --random-n); --profile-part solve puts only the solve, with --profile-nrhs
    right-hand sides, in the range; --profile-precision the Schur-update arithmetic (FPLUS_B200_PREC_*)."""
    import torch
    import fplus_b200 as F
    from fplus_b200 import workloads as W
    torch.cuda.init()
    if args.profile_workload == "stencil3d":
        n, Ap, Ai, Ax = W.convdiff3d(args.precision_grid, 3)
        desc = {"workload": f"3D convection-diffusion 7-point, {args.precision_grid}^3 grid (n={n}), float64"}
    elif args.profile_workload == "random":
        n, Ap, Ai, Ax = W.random_scaled(n=args.random_n)
        desc = {"workload": f"random complex base, scales over 17 decades (n={n})"}
    else:
        n, Ap, Ai, Ax, _, desc = workload(args.workload, args.modes)
    nrhs = args.profile_nrhs
    B = torch.from_numpy(W.rhs(n, nrhs, np.iscomplexobj(Ax), 2)).cuda()
    Ad = torch.from_numpy(np.ascontiguousarray(Ax)).cuda()
    S = F.analyze(n, Ap, Ai)
    if args.front_variant:
        S.set_front_shape(256, 64, args.front_variant)
    N = S.factor(Ad, device=True, precision=args.profile_precision)
    N.solve_device(B.clone(), 0)
    del N
    torch.cuda.synchronize()
    F.profile(True)
    solve_only = args.profile_part == "solve"
    if not solve_only:
        torch.cuda.cudart().cudaProfilerStart()
    N = S.factor(Ad, device=True, precision=args.profile_precision)
    Bc = B.clone()
    torch.cuda.synchronize()
    if solve_only:
        torch.cuda.cudart().cudaProfilerStart()
    N.solve_device(Bc, 0)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    prof = {F.PROFILE_CLASSES[c]: F.profile_read(c) for c in F.PROFILE_CLASSES}
    F.profile(False)
    desc.update({"n": n, "nrhs": nrhs, "part": args.profile_part, "precision": args.profile_precision})
    print(json.dumps({"profile_once": desc, "classes": prof}))


def traffic_ratio(kernel_class):
    """DRAM bytes per algorithmic byte of a kernel class's launches, from profiles/traffic.json (the ratio measured by an
    ncu capture of that kernel; the capture's summary is named there), or (None, reason)."""
    try:
        t = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))["classes"].get(kernel_class)
    except (OSError, ValueError, KeyError):
        return None, "profiles/traffic.json absent"
    if not t:
        return None, "no ncu capture of this class"
    return float(t["dram_to_algorithmic_bytes"]), f"{t['summary']} (ncu dram__bytes_read.sum + dram__bytes_write.sum)"


def run_precision_form(stream, dev, g=80, reps=2):
    """The precision form on the 3D convection-diffusion stencil (g^3 unknowns; g = 80: n = 512,000, the precision
    configuration): for each Schur-update arithmetic (FP64 = the plain form, FP32 = split TF32 x3, BF16X3, TF32), the
    device time of the factorization (values resident in HBM) and of the refined solve to a componentwise backward
    error of 1e-14 (classic refinement, GMRES-IR where it stalls; host right-hand side in and solution out), the normwise
    backward error, the forward difference from the FP64 solution, and the tensor-core share of the factorization's flops.
    Timed on the library's stream with CUDA events, median of `reps` after one warm-up each."""
    import torch
    import fplus_b200 as F
    import oracle as O
    from fplus_b200 import workloads as W
    t0 = time.perf_counter()
    n, Ap, Ai, Ax = W.convdiff3d(g, 3)
    S = F.analyze(n, Ap, Ai)
    analyze_ms = (time.perf_counter() - t0) * 1e3
    b = W.rhs(n, 1, False, 2)[0]
    Ad = torch.from_numpy(Ax).to(dev)
    out = {"workload": f"3D convection-diffusion 7-point, {g}^3 grid (n={n}, {int(Ap[-1])} entries), float64, nrhs 1",
           "analyze_ms": round(analyze_ms, 1), "forms": {}}
    x64 = None
    names = {F.PREC_FP64: "fp64", F.PREC_FP32: "fp32_split_tf32x3", F.PREC_BF16X3: "bf16x3", F.PREC_TF32: "tf32"}
    for prec in (F.PREC_FP64, F.PREC_FP32, F.PREC_BF16X3, F.PREC_TF32):
        rec = {"factor_ms": [], "solve_ms": []}
        for r in range(reps + 1):
            torch.cuda.synchronize()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            N = S.factor(Ad, device=True, precision=prec)
            e1.record(stream)
            x, berr, it = N.solve_refine(b, 0, max_iter=40, tol=1e-14)
            e2.record(stream)
            e2.synchronize()
            if r > 0:
                rec["factor_ms"].append(e0.elapsed_time(e1))
                rec["solve_ms"].append(e1.elapsed_time(e2))
            info = N.info
            del N
        f_ms, s_ms = float(np.median(rec["factor_ms"])), float(np.median(rec["solve_ms"]))
        be = O.backward_error(n, Ap, Ai, Ax, x, b)
        if prec == F.PREC_FP64:
            x64 = x.copy()
        d = {"factor_ms": f_ms, "refined_solve_ms": s_ms, "total_ms": f_ms + s_ms, "corrections": int(it[0]),
             "berr_componentwise": float(berr[0]), "berr": be,
             "forward_diff_vs_fp64": float(np.linalg.norm(x - x64) / np.linalg.norm(x64)),
             "tc_updates": int(info["tc_updates"]), "tc_flop_share": float(info["tc_flops"] / max(info["front_flops"], 1.0)),
             "front_flops": info["front_flops"], "device_GB": round(info["device_bytes"] / 1e9, 2)}
        if prec != F.PREC_FP64:
            # the Schur class's device time in one profiled factorization: the tensor-core updates' algorithmic rate
            F.profile(True)
            N = S.factor(Ad, device=True, precision=prec)
            torch.cuda.synchronize()
            pr = F.profile_read(0)
            F.profile(False)
            del N
            d["schur_ms"] = pr["ms"]
            d["schur_tflops_fp64_equivalent"] = pr["flops"] / max(pr["ms"], 1e-9) / 1e9
        out["forms"][names[prec]] = d
    base = out["forms"]["fp64"]["total_ms"]
    for k, v in out["forms"].items():
        v["speedup_vs_fp64"] = base / v["total_ms"] if v["berr"] <= 1e-14 else None
    ok = [v["total_ms"] for k, v in out["forms"].items() if k != "fp64" and v["berr"] <= 1e-14]
    out["best_mixed_speedup_vs_plain"] = base / min(ok) if ok else None
    return out


def run_random_form(stream, dev, n=40000, nrhs=256, reps=1):
    """C5, the ill-conditioned stress configuration, at n = `n`: the seeded well-conditioned random complex base (12
    entries per column) scaled by row and column factors over 17 decades, Ruiz on, `nrhs` right-hand sides solved
    together.  The plain form (FP64 Schur updates) against the FP32 form (split TF32x3 on the tensor cores) with FP64
    refinement (classic, GMRES-IR where it stalls) to a componentwise backward error of 1e-14 for every right-hand side.
    Device time of the factorization (values in HBM) and of the refined solve (host right-hand sides in, solutions out),
    CUDA events on the library's stream, median of `reps` after one warm-up.  The specified n = 300,000 does not fit:
    the static front structure of this random pattern holds about 0.85 n^2 entries."""
    import torch
    import fplus_b200 as F
    import oracle as O
    from fplus_b200 import workloads as W
    nn, Ap, Ai, Ax = W.random_scaled(n=n)
    S = F.analyze(nn, Ap, Ai)
    B = W.rhs(nn, nrhs, True, 5).T.copy(order="F")
    Ad = torch.from_numpy(Ax).to(dev)
    out = {"workload": f"random complex base, 12 entries per column, row / column scales over 17 decades (n={nn}, "
                       f"{int(Ap[-1])} entries), {nrhs} right-hand sides", "forms": {}}
    X64 = None
    for prec, name in ((F.PREC_FP64, "fp64"), (F.PREC_FP32, "fp32_split_tf32x3")):
        fms, sms = [], []
        for r in range(reps + 1):
            torch.cuda.synchronize()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            N = S.factor(Ad, device=True, precision=prec)
            e1.record(stream)
            X, berr, it = N.solve_refine(B, 0, max_iter=40, tol=1e-14)
            e2.record(stream)
            e2.synchronize()
            if r > 0:
                fms.append(e0.elapsed_time(e1)); sms.append(e1.elapsed_time(e2))
            info = N.info
            del N
        be = max(O.backward_error(nn, Ap, Ai, Ax, X[:, c], B[:, c]) for c in (0, nrhs // 2, nrhs - 1))
        if prec == F.PREC_FP64:
            X64 = X.copy()
        f_ms, s_ms = float(np.median(fms)), float(np.median(sms))
        out["forms"][name] = {"factor_ms": f_ms, "refined_solve_ms": s_ms, "total_ms": f_ms + s_ms,
                              "corrections_max": int(it.max()), "berr_componentwise_max": float(berr.max()),
                              "berr_normwise_sampled": be,
                              "forward_diff_vs_fp64": float(np.linalg.norm(X - X64) / np.linalg.norm(X64)),
                              "tc_flop_share": float(info["tc_flops"] / max(info["front_flops"], 1.0)),
                              "device_GB": round(info["device_bytes"] / 1e9, 2)}
    f = out["forms"]
    ok = f["fp32_split_tf32x3"]["berr_componentwise_max"] <= 1e-14
    out["speedup_fp32_vs_fp64"] = f["fp64"]["total_ms"] / f["fp32_split_tf32x3"]["total_ms"] if ok else None
    return out


def run_shift_batch(S, n, modes, count, b, wave=8):
    """count shifts A - sigma_k B (sigma_k = 0.3 + 1.7i + 0.1 k) of the benchmark pencil on its one analysis, nrhs 1:
    factored and solved through fplus_b200_factor_batch / solve_batch in waves of `wave` matrices (each factorization of
    this pencil holds about 9 GB of device memory), against the same calls one matrix at a time on the first `wave`
    shifts.  Device time: fplus_b200_batch_span_ms (CUDA events on the jobs' own streams, from the first factorization's
    start to the last solve's end), summed over the waves."""
    import fplus_b200 as F
    import oracle as O
    from fplus_b200 import workloads as W
    _, Ap, Ai, A0 = W.pencil(modes=modes, sigma=0.0)
    Bv = A0 - W.pencil(modes=modes, sigma=1.0)[3]           # B's values on A's pattern (the pencil is linear in sigma)
    sig = [0.3 + 1.7j + 0.1 * k for k in range(count)]
    seq = []
    for k in range(min(wave, count) + 1):
        N = S.factor(A0 - sig[k % count] * Bv)
        N.solve(b)
        if k > 0:                                        # the first one warms up
            seq.append(F.batch_span_ms([N]))
        del N
    F.solve_batch(F.factor_batch([S] * 2, [A0 - sig[0] * Bv, A0 - sig[1] * Bv]), [b, b])     # warm-up of the workers
    spans, be, wall = [], 0.0, 0.0
    for w0 in range(0, count, wave):
        ks = list(range(w0, min(count, w0 + wave)))
        Axs = [A0 - sig[k] * Bv for k in ks]
        t0 = time.perf_counter()
        Ns = F.factor_batch([S] * len(ks), Axs, nworkers=len(ks))
        Xs = F.solve_batch(Ns, [b] * len(ks), nworkers=len(ks))
        wall += time.perf_counter() - t0
        spans.append(F.batch_span_ms(Ns))
        be = max(be, max(O.backward_error(n, Ap, Ai, Axs[i], Xs[i], b) for i in range(len(ks))))
        del Ns
    dev = float(sum(spans))
    one = float(np.median(seq))
    return {"workload": f"{count} shifts sigma_k = 0.3+1.7i+0.1k of the benchmark pencil (n={n}), one analysis, nrhs 1, "
                        f"in waves of {wave}", "device_ms_total": dev, "device_ms_per_matrix": dev / count,
            "one_by_one_device_ms_per_matrix": one, "speedup_per_matrix": one / (dev / count), "berr_max": be,
            "host_wall_ms_total": wall * 1e3,
            "timing": "CUDA events on the jobs' streams (fplus_b200_batch_span_ms); values and right-hand sides from host memory"}


def run_pencil_batch(count, nworkers=32):
    """count independent pencils of uneven size (n log-uniform in [500, 8000], 2-4 dense tau rows / columns), 8
    right-hand sides each: analysed once each (not timed), then factored and solved one by one and through
    fplus_b200_factor_batch / solve_batch.  Device time from CUDA events on the jobs' own streams
    (fplus_b200_batch_span_ms); the one-by-one figure is the sum of each matrix's own span."""
    from concurrent.futures import ThreadPoolExecutor
    import fplus_b200 as F
    import oracle as O
    from fplus_b200 import workloads as W
    mats = W.pencil_batch(count=count)
    with ThreadPoolExecutor(16) as ex:
        syms = list(ex.map(lambda m: F.analyze(m[0], m[1], m[2]), mats))
    rhs = [W.rhs(m[0], 8, True, 7 + k).T.copy(order="F") for k, m in enumerate(mats)]
    F.solve_batch(F.factor_batch(syms[:4], [m[3] for m in mats[:4]]), rhs[:4])        # warm-up (and the dense-chain starts)
    # every pattern factored once, so that a restart for a dense-row pivot is not part of either timing
    for S, m in zip(syms, mats):
        S.factor(m[3])
    seq = 0.0
    t0 = time.perf_counter()
    for S, m, b in zip(syms, mats, rhs):
        N = S.factor(m[3])
        N.solve(b)
        seq += F.batch_span_ms([N])
        del N
    seq_wall = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    Ns = F.factor_batch(syms, [m[3] for m in mats], nworkers=nworkers)
    Xs = F.solve_batch(Ns, rhs, nworkers=nworkers)
    wall = (time.perf_counter() - t0) * 1e3
    dev = F.batch_span_ms(Ns)
    be = max(O.backward_error(m[0], m[1], m[2], m[3], X[:, r], b[:, r]) for m, X, b in zip(mats, Xs, rhs) for r in (0, 7))
    ns = [m[0] for m in mats]
    out = {"workload": f"{count} pencils, n log-uniform in [500, 8000] (sum {sum(ns)}), complex128, 8 right-hand sides each",
           "device_ms_total": dev, "one_by_one_device_ms_total": seq, "speedup": seq / dev, "berr_max": be,
           "workers": nworkers, "host_wall_ms_total": wall, "one_by_one_host_wall_ms_total": seq_wall,
           "timing": "CUDA events on the jobs' streams (fplus_b200_batch_span_ms); analysis excluded; values and right-hand "
                     "sides from host memory"}
    # the same step captured as one CUDA graph (every pencil an independent branch), replayed: the values and right-hand
    # sides uploaded, the graph launched, the statuses read and the solutions downloaded, inside CUDA events on the
    # launching stream (e2e), and the launch alone
    try:
        import torch
        st = torch.cuda.Stream()           # a stream of its own (the legacy default stream would not wait for the graph)
        G = F.BatchGraph(Ns, 8)
        def step():
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(st)
            for k, m in enumerate(mats):
                G.upload(k, m[3], rhs[k])
            e1.record(st)
            G.launch(st.cuda_stream)
            e2.record(st)
            rcs = G.status()
            Xg = [G.download(k) for k in range(len(mats))]
            t_end = torch.cuda.Event(enable_timing=True)
            t_end.record(st)
            t_end.synchronize()
            return e1.elapsed_time(e2), e0.elapsed_time(t_end), rcs, Xg
        step()
        runs = [step() for _ in range(3)]
        g_dev = float(np.median([r[0] for r in runs]))
        g_e2e = float(np.median([r[1] for r in runs]))
        rcs, Xg = runs[-1][2], runs[-1][3]
        beg = max(O.backward_error(m[0], m[1], m[2], m[3], X[:, r], b[:, r]) for m, X, b in zip(mats, Xg, rhs) for r in (0, 7))
        out["graph"] = {"device_ms_total": g_dev, "e2e_ms_total": g_e2e, "speedup_vs_one_by_one": seq / g_dev,
                        "statuses_ok": sum(1 for r in rcs if r == 0), "berr_max": beg,
                        "timing": "CUDA events on the launching stream: the graph launch alone (device), and uploads + launch "
                                  "+ status + downloads (e2e)"}
        del G
    except Exception as ex:                     # reported, not fatal: the uncaptured batch above stands
        out["graph"] = {"error": str(ex)[:300]}
    return out


def run_reference_arm(args, rank, world):
    """The reference's own CPU implementation on this arm's configuration (rank 0 only).  The 100 x 100 stencil runs in
    full.  The benchmark pencil (n = 32,768) does not finish within this arm's few-minute bound on the host cores: the arm
    times the reference on the same generator with 1 and 2 Fourier modes and prints the unavailable line with those
    measured times as the reason (no extrapolation)."""
    if rank != 0:
        return
    if not __import__("oracle").have_reference():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfplusref.so was not built (the reference "
                                                                "sources were absent at build time)"}))
        return
    from fplus_b200 import workloads as W
    threads = ref_threads()
    if args.workload == "pencil":
        t1, be1, n1 = reference_time("pencil_m1", lambda: W.pencil(modes=1), 1)
        t2, be2, n2 = reference_time("pencil_m2", lambda: W.pencil(modes=2), 1)
        print(json.dumps({"impl": "reference", "unavailable": (
            f"the reference's CPU factor+solve of the benchmark pencil (8 Fourier modes, n=32768) does not finish within "
            f"this arm's few-minute bound: measured here on {threads} host threads, the same generator took {t1:.0f} ms at "
            f"1 mode (n={n1}, berr {be1:.1e}) and {t2:.0f} ms at 2 modes (n={n2}, berr {be2:.1e}), {t2 / t1:.0f}x for 2x n"),
            "samples": {"pencil_m1": {"n": n1, "ms": t1, "berr": be1}, "pencil_m2": {"n": n2, "ms": t2, "berr": be2},
                        "threads": threads}}))
        return
    gen = lambda: W.convdiff2d(100, 1)
    for _ in range(max(args.warmup, 0)):
        reference_time("convdiff2d_g100", gen, 1)
    ms, be, n = reference_time("convdiff2d_g100", gen, max(args.steps, 1))
    d = workload(args.workload, args.modes)[5]
    line = {"impl": "reference", "metric": "factor+solve ms (berr<=1e-14)", "value": ms, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": d,
            "cpu_baseline": {"value": ms, "unit": "ms", "cores": threads, "kind": "reference",
                             "sample": f"the full workload, median of {max(args.steps, 1)} factor+solve steps; berr {be:.2e}"},
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def reference_subprocess(workload_name, steps, threads=None):
    """bench.py --impl reference in a child process (so OMP_NUM_THREADS applies from the start); its JSON line."""
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    if threads:
        env["OMP_NUM_THREADS"] = env["OPENBLAS_NUM_THREADS"] = str(threads)
    out = subprocess.run([sys.executable, os.path.abspath(__file__), "--impl", "reference", "--workload", workload_name,
                          "--steps", str(steps), "--warmup", "1"], env=env, capture_output=True, text=True, timeout=900)
    for line in out.stdout.splitlines()[::-1]:
        if line.startswith("{"):
            return json.loads(line)
    return {"unavailable": (out.stderr or "no output")[-300:]}


def run_c1_pair(stream, dev, steps=10, warmup=3):
    """The 100 x 100 stencil (n = 10,000, the reference's CPU-runnable configuration) in full on both sides: this
    library's device and end-to-end times and the reference's CPU build at all host cores and at 1 thread, each its
    median over `steps` factor+solve steps, the analysis done once beforehand on both sides (the same orders)."""
    import torch
    import fplus_b200 as F
    import oracle as O
    from fplus_b200 import workloads as W
    n, Ap, Ai, Ax = W.convdiff2d(100, 1)
    b = W.rhs(n, 1, False, 2)[0]
    S = F.analyze(n, Ap, Ai)
    rp, cp, _, _ = load_orders("convdiff2d_g100", Ap, Ai)
    same_orders = bool(np.array_equal(S.row_perm, rp) and np.array_equal(S.col_perm, cp))
    Ad = torch.from_numpy(Ax).to(dev)
    bd0 = torch.from_numpy(b).to(dev)
    Ah = torch.from_numpy(Ax).pin_memory().numpy()
    bh = torch.from_numpy(b).pin_memory()

    def dev_step():
        bd = bd0.clone()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        N = S.factor(Ad, device=True)
        N.solve_device(bd, 0)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), bd

    def e2e_step():
        xb = bh.clone().numpy()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        N = S.factor(Ah)
        err = ctypes.create_string_buffer(512)
        rc = F.lib().fplus_solve(N._h, xb.ctypes.data_as(ctypes.c_void_p), 1, n, 0, err, 512)
        assert rc == 0, err.value
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), xb
    for _ in range(warmup):
        dev_step(); e2e_step()
    td, te = [], []
    for _ in range(steps):
        ms, bd = dev_step(); td.append(ms)
        ms, xe = e2e_step(); te.append(ms)
    berr = O.backward_error(n, Ap, Ai, Ax, bd.cpu().numpy(), b)
    berr_e2e = O.backward_error(n, Ap, Ai, Ax, xe, b)
    ref_all = reference_subprocess("convdiff2d", 5)
    ref_one = reference_subprocess("convdiff2d", 5, threads=1)
    out = {"workload": "2D convection-diffusion 5-point, 100x100 grid (n=10000, 49600 entries), float64, nrhs 1",
           "same_orders": same_orders, "gpu_ms": float(np.median(td)), "gpu_e2e_ms": float(np.median(te)),
           "berr": berr, "berr_e2e": berr_e2e, "steps": steps,
           "reference_ms_all_threads": ref_all.get("value"), "reference_threads": ref_all.get("cpu_baseline", {}).get("cores"),
           "reference_ms_1_thread": ref_one.get("value"),
           "reference_berr": ref_all.get("cpu_baseline", {}).get("sample")}
    best = [v for v in (ref_all.get("value"), ref_one.get("value")) if v]
    if best:
        out["reference_ms_best"] = min(best)
        out["e2e_speedup_vs_reference_best"] = min(best) / out["gpu_e2e_ms"]
    return out


def run_b200_arm(args, rank, world):
    import torch
    import fplus_b200 as F
    import oracle as O
    from fplus_b200 import workloads as W

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n, Ap, Ai, Ax, b, desc = workload(args.workload, args.modes)
    cplx = np.iscomplexobj(Ax)
    t0 = time.perf_counter()
    S = F.analyze(n, Ap, Ai)
    analyze_ms = (time.perf_counter() - t0) * 1e3
    # one stream for the library's work, torch's work and the timing events (not the legacy default stream, which the
    # library's own non-blocking streams would not be ordered with)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    F.lib().fplus_b200_use_stream(ctypes.c_void_p(stream.cuda_stream))
    # the front shape for this pattern, picked once by the library's autotuner (untimed, like the analysis)
    t0 = time.perf_counter()
    if args.front_variant:
        S.set_front_shape(256, 64, args.front_variant)
    tuned = S.autotune(Ax) if not (args.no_autotune or args.front_variant) else None
    autotune_ms = (time.perf_counter() - t0) * 1e3
    Ad = torch.from_numpy(Ax).to(dev)
    bd0 = torch.from_numpy(np.ascontiguousarray(b)).to(dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def dev_step():
        bd = bd0.clone()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        N = S.factor(Ad, device=True)
        N.solve_device(bd, 0)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), N, bd

    for _ in range(args.warmup):
        _, N, _ = dev_step()
        del N
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    L0 = F.launch_count()
    times = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ms, N, bd = dev_step()
            times.append(ms)
            del N
    torch.cuda.synchronize()
    launches = F.launch_count() - L0
    ms_dev = allreduce_max(float(np.mean(times)), dev)
    x = bd.cpu().numpy()
    berr = O.backward_error(n, Ap, Ai, Ax, x, b)

    # e2e: the public host API with pinned buffers
    Ah = torch.from_numpy(Ax).pin_memory()
    bh = torch.from_numpy(np.ascontiguousarray(b)).pin_memory()
    Ah_np = Ah.numpy()

    def e2e_step():
        xb = bh.clone()              # pinned, solved in place
        xb_np = xb.numpy()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        err = ctypes.create_string_buffer(512)
        h = ctypes.c_void_p()
        rc = F.lib().fplus_factor(S._h, F._p64(S.Ap), F._p64(S.Ai), Ah_np.ctypes.data_as(ctypes.c_void_p), int(cplx),
                                  ctypes.byref(S.options), ctypes.byref(h), err, 512)
        assert rc == 0, err.value
        rc = F.lib().fplus_solve(h, xb_np.ctypes.data_as(ctypes.c_void_p), 1, n, 0, err, 512)
        assert rc == 0, err.value
        e1.record(stream)
        e1.synchronize()
        F.lib().fplus_numeric_free(h)
        return e0.elapsed_time(e1), xb_np
    for _ in range(min(args.warmup, 2)):
        e2e_step()
    e2e_times = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ms, xe = e2e_step()
        e2e_times.append(ms)
    ms_e2e = allreduce_max(float(np.mean(e2e_times)), dev)
    berr_e2e = O.backward_error(n, Ap, Ai, Ax, xe, b)
    vsz = 16 if cplx else 8

    # roofline: one profiled step, the dominant class
    F.profile(True)
    flush.zero_()
    _, N, _ = dev_step()
    info = N.info
    del N
    prof = {F.PROFILE_CLASSES[c]: F.profile_read(c) for c in F.PROFILE_CLASSES}
    F.profile(False)
    dom = max(prof, key=lambda k: prof[k]["ms"])
    peaks, psrc = measured_peaks()
    fp64_peak = fp64_peak_tflops(torch, cplx) if rank == 0 else float("nan")

    def class_roofline(cls):
        p = prof[cls]
        if cls == "assemble":
            achieved = p["bytes"] / (p["ms"] * 1e-3) / 1e9
            r = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                 "frac": achieved / peaks["hbm_gbs"], "peak_source": f"hbm_gbs ({psrc})"}
        else:
            achieved = p["flops"] / (p["ms"] * 1e-3) / 1e12
            r = {"bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                 "peak_source": ("cuBLAS " + ("ZGEMM" if cplx else "DGEMM") + " 8192^3 measured in bench.py (FP64 tensor "
                                 "path; the measured-peaks file has bf16 and HBM only)")}
        ratio, rsrc = traffic_ratio(cls)
        r.update({"kernel_class": cls, "launches": p["count"], "avg_launch_us": 1e3 * p["ms"] / max(p["count"], 1),
                  "algorithmic_per_launch": (p["flops"] if cls != "assemble" else p["bytes"]) / max(p["count"], 1),
                  "algorithmic_bytes_per_launch": p["bytes"] / max(p["count"], 1),
                  "traffic": None if ratio is None else ratio * p["bytes"] / max(p["count"], 1),
                  "traffic_source": rsrc})
        return r
    roof = class_roofline(dom)
    roof["classes_ms"] = {k: round(v["ms"], 3) for k, v in prof.items()}
    if dom == "front_lu":
        # the pivot-block LU is bound by the latency of its dependent pivot steps, not by a throughput; the Schur
        # updates' roofline beside it
        roof["bound_note"] = "latency of np dependent pivot steps per front (one CTA); no throughput roofline applies"
    roof_schur = class_roofline("schur_gemm") if dom != "schur_gemm" and prof["schur_gemm"]["count"] > 0 else None

    # the solve with 16 right-hand sides (the configuration's second nrhs)
    solve16 = None
    if args.workload == "pencil":
        N16 = S.factor(Ad, device=True)
        B16 = torch.from_numpy(W.rhs(n, 16, cplx, 5)).to(dev)       # (16, n): column-major n x 16
        N16.solve_device(B16.clone(), 0)
        ts = []
        for _ in range(3):
            Bc = B16.clone()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            N16.solve_device(Bc, 0)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        X16 = Bc.cpu().numpy().T
        B16h = B16.cpu().numpy().T
        be16 = max(O.backward_error(n, Ap, Ai, Ax, X16[:, r], B16h[:, r]) for r in range(16))
        solve16 = {"nrhs": 16, "ms": float(np.median(ts)), "berr_max": be16}
        del N16

    # the batch form: shifts sigma_k of the same pencil on one analysis, factored and solved concurrently
    batch = None
    if args.workload == "pencil" and args.batch > 0 and world == 1:
        batch = run_shift_batch(S, n, args.modes, args.batch, b)
    batch_pencils = None
    if args.batch_pencils > 0 and world == 1:
        batch_pencils = run_pencil_batch(args.batch_pencils)
    c1_pair = None
    if world == 1 and not args.no_cpu_baseline and __import__("oracle").have_reference():
        c1_pair = run_c1_pair(stream, dev)
    precision = None
    if world == 1 and args.precision_grid > 0:
        precision = run_precision_form(stream, dev, args.precision_grid)
    random_form = None
    if world == 1 and args.random_n > 0:
        random_form = run_random_form(stream, dev, args.random_n)

    if rank != 0:
        return
    clocks = clk.summary()
    cpu = None
    if __import__("oracle").have_reference() and world == 1 and not args.no_cpu_baseline:
        if args.workload == "pencil":
            ms_s, be_ref, n_s = reference_time("pencil_m1", lambda: W.pencil(modes=1), 3)
            cpu = {"value": ms_s, "unit": "ms", "cores": ref_threads(), "kind": "reference", "scaled": False,
                   "sample": (f"the same pencil generator with 1 Fourier mode (n={n_s}) instead of 8 (n={n}): the "
                              f"reference's factor+solve, median of 3, berr {be_ref:.2e}; measured, not scaled to n={n} "
                              "(the full size does not finish within minutes; c1_pair compares both in full on the "
                              "CPU-runnable configuration)")}
        else:
            ms_s, be_ref, n_s = reference_time("convdiff2d_g100", lambda: W.convdiff2d(100, 1), 5)
            cpu = {"value": ms_s, "unit": "ms", "cores": ref_threads(), "kind": "reference", "scaled": False,
                   "sample": f"the full workload, median of 5 factor+solve steps, berr {be_ref:.2e}"}
    line = {"metric": "factor+solve ms (berr<=1e-14)", "value": ms_dev / world, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_dev, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128" if cplx else "f64", "data": "synthetic",
            "config": dict(desc, **{"parallelism": f"replicas{world}" if world > 1 else "1 GPU",
                                    "l2": "flushed between steps (512 MiB write)", "analyze_ms": round(analyze_ms, 2),
                                    "front_variant": args.front_variant or None,
                                    "front_shape": None if tuned is None else {"max_width": tuned[0], "nb_chain": tuned[1],
                                                                                "lu_kernel": tuned[2],
                                                                                "autotune_ms": round(autotune_ms, 1)},
                                    "berr": berr, "berr_e2e": berr_e2e, "fronts": info["nfronts"],
                                    "dense_chain_from": info["f_dense"], "ms_equil": round(info["ms_equil"], 3),
                                    "ms_fronts": round(info["ms_fronts"], 3), "front_flops": info["front_flops"]}),
            "e2e": {"value": ms_e2e / world, "unit": "ms", "h2d_bytes_per_step": int(Ap[-1]) * vsz + n * vsz,
                    "d2h_bytes_per_step": n * vsz},
            "gpu_launches": int(launches),
            "clocks": clocks, "roofline": roof, "roofline_schur": roof_schur, "cpu_baseline": cpu, "solve_nrhs16": solve16, "batch": batch,
            "batch_pencils": batch_pencils, "c1_pair": c1_pair, "precision_form": precision, "random_form": random_form}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="pencil", choices=["pencil", "convdiff2d"])
    ap.add_argument("--modes", type=int, default=8,
                    help="Fourier modes of the pencil workload (8: n = 32768, the benchmark; 1: n = 4096, for profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default front shape (no fplus_b200_autotune)")
    ap.add_argument("--front-variant", type=int, default=0,
                    help="fplus_b200_set_front_shape variant for the benchmark pattern instead of the autotuner (0: autotune)")
    ap.add_argument("--precision-grid", type=int, default=80,
                    help="grid of the 3D stencil of the precision-form measurement (80: n = 512,000; 0: none)")
    ap.add_argument("--random-n", type=int, default=40000,
                    help="n of the 17-decade random configuration with 256 right-hand sides (0: none)")
    ap.add_argument("--batch", type=int, default=64, help="shifts of the pencil in the batch measurement (0: none)")
    ap.add_argument("--batch-pencils", type=int, default=512,
                    help="independent uneven pencils in the second batch measurement (0: none)")
    ap.add_argument("--profile-workload", default="bench", choices=["bench", "stencil3d", "random"])
    ap.add_argument("--profile-part", default="all", choices=["all", "solve"])
    ap.add_argument("--profile-nrhs", type=int, default=1)
    ap.add_argument("--profile-precision", type=int, default=0)
    ap.add_argument("--profile-once", action="store_true",
                    help="for ncu --profile-from-start off: one warm factorization, then exactly one factor + solve "
                         "between cudaProfilerStart / Stop; prints that factorization's algorithmic work per class")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and args.impl == "b200":
        import datetime
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.profile_once:
            run_profile_once(args)
        elif args.impl == "reference":
            run_reference_arm(args, rank, world)
        else:
            run_b200_arm(args, rank, world)
    finally:
        if world > 1 and args.impl == "b200":
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
