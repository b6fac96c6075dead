"""Benchmark: mixed-precision LU with FP64 iterative refinement against plain FP32 LU + solve,
on B200, through the aclsolver C ABI, with the plain batched factor-and-solve workloads
measured beside it.

Headline workload (the mixed-precision batched LU configuration): 256 matrices of order
512, A = U diag(s) V^T with U, V Haar-random orthogonal (QR of N(0,1)) and s log-spaced from
1 to 1/kappa, kappa cycling through 1e2, 1e4, 1e5 over the batch; one N(0,1) right-hand side
each.  All data is synthetic (seeded); no benchmark suite is involved.

One step = one aclsolverSgesvIrBatched call over the batch (split-BF16 tensor-core trailing
updates, FP32 panels and solves, FP64 residual and update, tolerance 1e-7 on the normwise
backward error).  `value` is solves/s of that call with the inputs resident in HBM (device
time from CUDA events on the handle stream, summed over the K timed steps; the inputs are
256 MiB, larger than the 126 MB L2, and a 256 MiB buffer is written before each step).  The
plain FP32 path (aclsolverSgetrfBatched + aclsolverSgetrsBatched, the reference's method) is
timed the same way and reported beside it with both backward errors (`plain`, `mixed`), so the
ratio is taken at equal (FP32-level) backward error.  `e2e` is the refinement call with
pinned host buffers: A and b copied in and x copied out inside the timed region.

`configs` carries the plain batched workloads, each timed on the device the same way (inputs
restored from a pristine copy and a 256 MiB buffer written before every step, so the timed
bytes come from HBM) with its roofline and its own CPU baseline:
  c1  10,000 SPD 32x32, SpotrfBatched + SpotrsBatched (fp32, lower, 1 RHS);
  c2  4,096 N(0,1) 64x64, SgetrfBatched + SgetrsBatched + SgetriBatched (fp32, 1 RHS);
  c3  20,000 HPD complex64 of orders U{8..128}, 4 RHS, one CposvVbatched call (persistent,
      size-bucketed, graph-captured, autotuned).
`large` carries the single 8192 x 8192 system (plain and mixed).

CPU baseline: the host LAPACK the reference's tests use as their golden (scipy's bundled
OpenBLAS, FP32 sgetrf/sgetrs/sgetri/spotrf/spotrs/cpotrf/cpotrs) on this host's cores, OpenMP
over matrices with one OpenBLAS thread per call (OpenBLAS threaded for the single system).

`python bench.py --impl reference` times that same host LAPACK on the headline workload (all
256 systems, the same step count).

Multi-GPU (`torchrun ... bench.py --gpus N`): every rank solves its own batch of 256 systems
(independent matrices: replicas, no data-path collective); time is the maximum over ranks and
`value` the solves of all ranks over that time.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "ops-solver_b200"))

COUNT = 256
N = 512
NRHS = 1
KAPPAS = (1e2, 1e4, 1e5)
TOL = 1e-7
MAX_ITER = 4
PRECISION = 3  # ACLSOLVER_FACTOR_BF16X3
METRIC = "solves/s & GFLOP/s: mixed-prec+IR vs plain FP32, same B200, equal backward error"
UNIT = "solves/s"
WORKLOAD = ("mixed-precision batched LU + FP64 iterative refinement vs plain FP32 sgetrf/sgetrs: "
            "256 x 512x512, A = U diag(s) V^T, kappa in {1e2, 1e4, 1e5}, 1 RHS")
# Nominal work of one solve (LU 2n^3/3 + two triangular solves 2n^2) for GFLOP/s, and the
# algorithmic bytes of one launch of the dominant kernel (the batched factorisation: reads
# and writes its n x n working copy once).
SOLVE_FLOPS = 2 * N**3 / 3 + 2 * N * N * NRHS
FACTOR_BYTES = 2 * N * N * 4
FACTOR_FLOPS = 2 * N**3 / 3
FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
SMS = 148
FLUSH_BYTES = 256 << 20


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return FALLBACK["hbm_gbs"], FALLBACK["bf16_tflops"], "fallback"


def fp32_peak_tflops():
    """FP32 FMA peak of the chip at its maximum SM clock: 148 SMs x 128 lanes x 2 flops.
    No measured FP32 figure exists for this pool, so this one is nominal."""
    mhz = 1965.0
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        mhz = float(json.loads(p.read_text()).get("sm_max_mhz", mhz))
    return SMS * 128 * 2 * mhz * 1e6 / 1e12


def traffic_summary():
    """Per-launch DRAM bytes of the dominant kernels from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            return {}
    return {}


def roofline(bytes_, flops, ms, kernel, traffic_key=None):
    """Roofline of one timed region: the floor is the slower of the algorithmic bytes at the
    measured HBM bandwidth and the flops at the FP32 FMA peak; `frac` is achieved / peak on
    the bound that sets the floor."""
    hbm, _, kind = peaks()
    fp32 = fp32_peak_tflops()
    t_hbm = bytes_ / (hbm * 1e9) * 1e3
    t_fp32 = flops / (fp32 * 1e12) * 1e3
    gbs = bytes_ / (ms * 1e-3) / 1e9
    tflops = flops / (ms * 1e-3) / 1e12
    out = {"kernel": kernel}
    if t_hbm >= t_fp32:
        out.update({"bound": "hbm", "achieved": round(gbs, 1), "peak": hbm, "unit": "GB/s",
                    "frac": round(gbs / hbm, 4), "peak_kind": kind})
    else:
        out.update({"bound": "fp32", "achieved": round(tflops, 2), "peak": round(fp32, 1), "unit": "TFLOP/s",
                    "frac": round(tflops / fp32, 4), "peak_kind": "nominal FP32 FMA at the max SM clock"})
    out.update({"hbm_frac": round(gbs / hbm, 4), "fp32_frac": round(tflops / fp32, 4),
                "floor_ms": round(max(t_hbm, t_fp32), 5), "measured_ms": round(ms, 5),
                "floor_over_measured": round(max(t_hbm, t_fp32) / ms, 4),
                "algorithmic_bytes": int(bytes_), "algorithmic_flops": int(flops),
                "traffic": traffic_summary().get(traffic_key) if traffic_key else None})
    return out


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    QUERY = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader",
                 "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            time.sleep(0.3)  # the first sample lands before the timed work starts
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.05)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                mx = float(f[2].split()[0])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def make_inputs(seed, count=COUNT):
    """Column-major slabs of `count` conditioned matrices and right-hand sides."""
    import numpy as np

    rng = np.random.default_rng(seed)
    a = np.empty((count, N, N), dtype=np.float32)
    for q in range(count):
        kappa = KAPPAS[q % len(KAPPAS)]
        s = np.logspace(0.0, -np.log10(kappa), N)
        u, ru = np.linalg.qr(rng.standard_normal((N, N)))
        v, rv = np.linalg.qr(rng.standard_normal((N, N)))
        u *= np.sign(np.diag(ru))
        v *= np.sign(np.diag(rv))
        a[q] = ((u * s) @ v.T).astype(np.float32)
    b = rng.standard_normal((count, N, NRHS)).astype(np.float32)
    return a, b


def colmajor(x):
    import numpy as np

    return np.ascontiguousarray(x.transpose(0, 2, 1))


def backward_errors(a_cm, x_cm, b_cm, count, device):
    """Normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) per matrix,
    FP64 on the GPU (a check of the result, outside the timed region)."""
    import torch

    A = a_cm.view(count, N, N).transpose(1, 2).double()  # row-major view of column-major data
    X = x_cm.view(count, NRHS, N).transpose(1, 2).double()
    B = b_cm.view(count, NRHS, N).transpose(1, 2).double()
    R = B - torch.bmm(A, X)
    num = R.abs().amax(dim=(1, 2))
    den = A.abs().sum(dim=2).amax(dim=1) * X.abs().amax(dim=(1, 2)) + B.abs().amax(dim=(1, 2))
    return (num / den).cpu().numpy()


def fp64_solutions(a, b):
    """FP64 LAPACK (numpy's gesv) solutions of every system: the forward-error oracle."""
    import numpy as np

    return np.linalg.solve(a.astype(np.float64), b.astype(np.float64))


def forward_errors(x64, x):
    """||x - x64||_inf / ||x64||_inf per system."""
    import numpy as np

    d = np.abs(x.astype(np.float64) - x64).max(axis=(1, 2))
    return d / np.abs(x64).max(axis=(1, 2))


class DeviceTimer:
    """Per-step device time of `fn` on `stream`: `before()` runs first (untimed: restore the
    inputs, then overwrite L2 with a 256 MiB buffer), then CUDA events bracket `fn`."""

    def __init__(self, stream, device):
        import torch

        self.torch = torch
        self.stream = stream
        self.flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=device)
        self.ev0 = torch.cuda.Event(enable_timing=True)
        self.ev1 = torch.cuda.Event(enable_timing=True)

    def __call__(self, fn, steps, before=None):
        torch = self.torch
        total = 0.0
        for i in range(steps):
            with torch.cuda.stream(self.stream):
                if before:
                    before()
                self.flush.fill_(i & 0xFF)
                self.ev0.record(self.stream)
                fn()
                self.ev1.record(self.stream)
            self.ev1.synchronize()
            total += self.ev0.elapsed_time(self.ev1)
        return total / max(1, steps)


def cpu_timed(fn, seconds, min_reps=2, max_reps=200):
    """Passes of `fn` for about `seconds` (at least `min_reps`); returns (s per pass, reps)."""
    fn()  # warm-up (page-in, thread pool start)
    reps, t0 = 0, time.perf_counter()
    while True:
        fn()
        reps += 1
        dt = time.perf_counter() - t0
        if (dt > seconds and reps >= min_reps) or reps >= max_reps:
            return dt / reps, reps


def run_b200(args, rank, world):
    import numpy as np
    import torch

    import aclsolver
    from aclsolver.shard import gather_to_root, shard_range

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    dev = torch.device("cuda", torch.cuda.current_device())
    lib = aclsolver.library()
    handle = aclsolver.Handle()
    aclsolver.check(lib.aclsolverSetDeviceChecks(handle.value, 0))
    stream = handle.stream

    # the global batch is COUNT systems per GPU, split into contiguous slices (one per rank,
    # no collective on the data path); each slice of COUNT systems is seeded by its index
    start, count = shard_range(COUNT * world, rank, world)
    assert count == COUNT
    a_host, b_host = make_inputs(1 + start // COUNT)
    a_cm, b_cm = colmajor(a_host), colmajor(b_host)
    A = torch.from_numpy(a_cm.reshape(-1)).to(dev)  # original matrices (read only)
    B = torch.from_numpy(b_cm.reshape(-1)).to(dev)
    X = torch.empty_like(B)
    W = torch.empty_like(A)  # plain path: factored in place
    XP = torch.empty_like(B)
    ta = aclsolver.pointer_table(A, COUNT, N * N * 4)
    tb = aclsolver.pointer_table(B, COUNT, N * NRHS * 4)
    tx = aclsolver.pointer_table(X, COUNT, N * NRHS * 4)
    tw = aclsolver.pointer_table(W, COUNT, N * N * 4)
    txp = aclsolver.pointer_table(XP, COUNT, N * NRHS * 4)
    piv = torch.empty(COUNT * N, dtype=torch.int32, device=dev)
    info = torch.empty(COUNT, dtype=torch.int32, device=dev)
    info_s = torch.empty(COUNT, dtype=torch.int32, device=dev)
    iters = torch.empty(COUNT, dtype=torch.int32, device=dev)
    berr = torch.empty(COUNT, dtype=torch.float64, device=dev)
    timer = DeviceTimer(stream, dev)
    # kernels launched by one refinement call: two pointer tables, the factorisation (with the
    # copy of A and the permutation) and its later-interchange pass, the diagonal-block
    # inverses, init, solve, update, MAX_ITER x (residual, solve, update), residual, finish
    launches_ir = 8 + 3 * MAX_ITER + 2

    def mixed(tables=None):
        a_t, b_t, x_t = tables or (ta, tb, tx)
        aclsolver.check(lib.aclsolverSgesvIrBatched(handle.value, PRECISION, N, NRHS, a_t.data_ptr(), N,
                                                    b_t.data_ptr(), N, x_t.data_ptr(), N, MAX_ITER, TOL,
                                                    iters.data_ptr(), berr.data_ptr(), info.data_ptr(), COUNT))

    def plain():
        aclsolver.check(lib.aclsolverSgetrfBatched(handle.value, N, tw.data_ptr(), N, piv.data_ptr(),
                                                   info.data_ptr(), COUNT))
        aclsolver.check(lib.aclsolverSgetrsBatched(handle.value, 0, N, NRHS, tw.data_ptr(), N, piv.data_ptr(),
                                                   txp.data_ptr(), N, info_s.data_ptr(), COUNT))

    def factor_only():
        aclsolver.check(lib.aclsolverSgetrfBatchedMixed(handle.value, PRECISION, N, tw.data_ptr(), N,
                                                        piv.data_ptr(), info.data_ptr(), COUNT))

    def restore():
        W.copy_(A)
        XP.copy_(B)

    for _ in range(args.warmup):
        timer(mixed, 1)
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0, "unexpected info"
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        wall0 = time.perf_counter()
        ms = timer(mixed, args.steps)
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
    barrier(world)
    ms = max_over_ranks(ms, world)
    mixed_berr = backward_errors(A, X, B, COUNT, dev)
    mixed_info = info.cpu().numpy()
    mixed_iters = iters.cpu().numpy()
    x_mixed = X.cpu().numpy().reshape(COUNT, NRHS, N).transpose(0, 2, 1)

    # plain FP32 path, same inputs (its working copy restored outside the timed region)
    for _ in range(max(3, args.warmup // 2)):
        timer(plain, 1, restore)
    plain_ms = max_over_ranks(timer(plain, max(3, args.steps // 2), restore), world)
    assert int(info.abs().max()) == 0 and int(info_s.abs().max()) == 0
    plain_berr = backward_errors(A, XP, B, COUNT, dev)
    x_plain = XP.cpu().numpy().reshape(COUNT, NRHS, N).transpose(0, 2, 1)

    # the dominant kernel alone (the split-BF16 factorisation) for the roofline
    for _ in range(3):
        timer(factor_only, 1, restore)
    factor_ms = timer(factor_only, max(3, args.steps // 2), restore)

    # e2e: host buffers, copies inside the timed region
    a_pin = torch.from_numpy(a_cm.reshape(-1)).pin_memory()
    b_pin = torch.from_numpy(b_cm.reshape(-1)).pin_memory()
    x_pin = torch.empty(X.numel(), dtype=torch.float32).pin_memory()
    # as many steps as the device-timed leg: the pipeline's fill and drain (one solve) are
    # spread over the same number of steps
    e2e_steps = max(3, args.steps)
    # streamed: two sets of device buffers; step s copies its inputs (pinned host -> device) on a
    # copy stream while step s - 1 computes, then solves and reads its solutions back
    A2, B2, X2 = torch.empty_like(A), torch.empty_like(B), torch.empty_like(X)
    sets = [(A, B, X, (ta, tb, tx)),
            (A2, B2, X2, (aclsolver.pointer_table(A2, COUNT, N * N * 4), aclsolver.pointer_table(B2, COUNT, N * NRHS * 4),
                          aclsolver.pointer_table(X2, COUNT, N * NRHS * 4)))]
    x_pins = [x_pin, torch.empty(X.numel(), dtype=torch.float32).pin_memory()]
    copy_stream = torch.cuda.Stream()
    done = [torch.cuda.Event(), torch.cuda.Event()]
    copied = [torch.cuda.Event(), torch.cuda.Event()]

    def e2e_step(step):
        k = step % 2
        a_d, b_d, x_d, tables = sets[k]
        copy_stream.wait_event(done[k])  # buffer set k is free (its previous step has read back)
        with torch.cuda.stream(copy_stream):
            a_d.copy_(a_pin, non_blocking=True)
            b_d.copy_(b_pin, non_blocking=True)
            copied[k].record(copy_stream)
        stream.wait_event(copied[k])
        with torch.cuda.stream(stream):
            mixed(tables)
            x_pins[k].copy_(x_d, non_blocking=True)
            done[k].record(stream)

    for step in range(2):
        e2e_step(step)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    copy_stream.wait_event(e0)
    for step in range(e2e_steps):
        e2e_step(step)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, world)
    assert bool(np.isfinite(x_pins[0].numpy()).all()) and bool(np.isfinite(x_pins[1].numpy()).all())
    h2d = COUNT * N * N * 4 + COUNT * N * NRHS * 4
    d2h = COUNT * N * NRHS * 4
    del A2, B2, X2, sets, x_pins

    configs = None
    if rank != 0:
        args.cpu_seconds = 0.0  # CPU baselines are taken on rank 0 only
    if args.configs:
        configs = {
            "c1": measure_c1(handle, timer, args),
            "c2": measure_c2(handle, timer, args),
            "c3": measure_c3(handle, timer, args),
        }

    # per-system results of every slice, in global batch order, on rank 0 (outside the timing)
    global_berr = {"mixed": mixed_berr, "plain": plain_berr, "info": mixed_info}
    if world > 1:
        global_berr = {k: gather_to_root(v, COUNT * world) for k, v in global_berr.items()}
    if rank == 0:
        hbm, bf16, peak_kind = peaks()
        x64 = fp64_solutions(a_host, b_host)
        fe_mixed = forward_errors(x64, x_mixed)
        fe_plain = forward_errors(x64, x_plain)
        value = COUNT * world / (ms * 1e-3)
        plain_value = COUNT * world / (plain_ms * 1e-3)
        achieved = FACTOR_BYTES * COUNT / (factor_ms * 1e-3) / 1e9
        roof_ms = max(FACTOR_BYTES * COUNT / (hbm * 1e9), FACTOR_FLOPS * COUNT / (bf16 * 1e12)) * 1e3
        cpu = cpu_baseline_headline(args, a_cm, b_cm, x64)
        large = measure_large(handle, args) if args.large else None
        complex_lu = measure_complex_lu(handle, args) if args.complex_lu else None
        qr = measure_qr(handle, args) if args.complex_lu else None
        by_kappa = {}
        for k, kappa in enumerate(KAPPAS):
            idx = list(range(k, COUNT, len(KAPPAS)))
            by_kappa[f"{kappa:.0e}"] = {
                "mixed_berr_max": float(mixed_berr[idx].max()),
                "plain_berr_max": float(plain_berr[idx].max()),
                "mixed_ferr_max": float(fe_mixed[idx].max()),
                "plain_ferr_max": float(fe_plain[idx].max()),
                "iterations_max": int(mixed_iters[idx].max()),
            }
        line = {
            "metric": METRIC,
            "value": round(value, 1),
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "fp32 interface; bf16x3 tensor-core trailing updates, fp32 panels/solves, fp64 residual",
            "data": "synthetic: seeded U diag(s) V^T matrices and N(0,1) right-hand sides",
            "config": {
                "workload": WORKLOAD,
                "batch_per_gpu": COUNT,
                "n": N,
                "nrhs": NRHS,
                "kappa": list(KAPPAS),
                "path": "aclsolverSgesvIrBatched(BF16X3, tol 1e-7, maxIter 4) vs SgetrfBatched + SgetrsBatched",
                "l2": "inputs 256 MiB (> L2) and a 256 MiB buffer written before each step",
                "parallelism": f"batch split over {world} GPU(s): {COUNT * world} systems, contiguous slices of "
                               f"{COUNT}, no data-path collective",
            },
            "global_batch": {"systems": COUNT * world,
                             "mixed_berr_max": float(global_berr["mixed"].max()),
                             "plain_berr_max": float(global_berr["plain"].max()),
                             "info_nonzero": int((global_berr["info"] != 0).sum())},
            "gflops": round(value * SOLVE_FLOPS / 1e9, 1),
            "mixed": {
                "solves_per_s": round(value, 1),
                "ms": round(ms, 4),
                "berr_max": float(mixed_berr.max()),
                "berr_reported_max": float(berr.max().item()),
                "iterations_max": int(mixed_iters.max()),
                "ferr_vs_fp64_max": float(fe_mixed.max()),
                "ferr_systems": COUNT,
            },
            "plain": {
                "solves_per_s": round(plain_value, 1),
                "ms": round(plain_ms, 4),
                "gflops": round(plain_value * SOLVE_FLOPS / 1e9, 1),
                "berr_max": float(plain_berr.max()),
                "ferr_vs_fp64_max": float(fe_plain.max()),
                "ferr_systems": COUNT,
            },
            "mixed_over_plain": round(value / plain_value, 3),
            "by_kappa": by_kappa,
            "roofline": {
                "kernel": "getrf_blocked_kernel<3> (split-BF16 batched LU)",
                "bound": "hbm",
                "achieved": round(achieved, 1),
                "peak": hbm,
                "peak_kind": peak_kind,
                "unit": "GB/s",
                "frac": round(achieved / hbm, 4),
                "traffic": traffic_summary().get("getrf_blocked_bf16x3"),
                "algorithmic_bytes_per_launch": FACTOR_BYTES * COUNT,
                "kernel_ms": round(factor_ms, 4),
                "roofline_ms": round(roof_ms, 4),
                "tensor_tflops_achieved": round(FACTOR_FLOPS * COUNT / (factor_ms * 1e-3) / 1e12, 2),
            },
            "e2e": {
                "value": round(COUNT * world / (e2e_ms * 1e-3), 1),
                "unit": UNIT,
                "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "ms_per_step": round(e2e_ms, 4),
                "mode": "streamed: each step copies its A and b from pinned host memory on a copy stream "
                        "while the previous step solves, then reads its X back (two device buffer sets)",
            },
            "gpu_launches": launches_ir * args.steps,
            "clocks": clocks.summary(),
            "wall_s_timed": round(wall, 4),
            "cpu_baseline": cpu,
            "configs": configs,
            "large": large,
            "complex_lu": complex_lu,
            "qr": qr,
        }
        print(json.dumps(line), flush=True)
    handle.close()


# ---------------------------------------------------------------------------------------
# The plain batched workloads (configs 1-3)
# ---------------------------------------------------------------------------------------

def measure_c1(handle, timer, args):
    """10,000 SPD matrices of order 32, A = G G^T / 32 + I (G ~ N(0,1), seed 0), lower,
    lda 32, one N(0,1) right-hand side: SpotrfBatched + SpotrsBatched."""
    import numpy as np
    import torch

    import aclsolver
    from oracle import host_lapack

    lib, check = aclsolver.library(), aclsolver.check
    count, n, nrhs = 10_000, 32, 1
    rng = np.random.default_rng(0)
    g = rng.standard_normal((count, n, n), dtype=np.float32)
    a = (np.matmul(g, g.transpose(0, 2, 1)) / n + np.eye(n, dtype=np.float32)).astype(np.float32)
    b = rng.standard_normal((count, n, nrhs), dtype=np.float32)
    a_cm, b_cm = colmajor(a).reshape(-1), colmajor(b).reshape(-1)
    A0 = torch.from_numpy(a_cm).cuda()
    B0 = torch.from_numpy(b_cm).cuda()
    A, B = torch.empty_like(A0), torch.empty_like(B0)
    ta, tb = aclsolver.pointer_table(A, count, n * n * 4), aclsolver.pointer_table(B, count, n * nrhs * 4)
    info = torch.empty(count, dtype=torch.int32, device="cuda")
    # SpotrsBatched reports through info[0] but, as the reference, takes batchSize entries
    sinfo = torch.empty(count, dtype=torch.int32, device="cuda")
    h = handle.value

    def potrf():
        check(lib.aclsolverSpotrfBatched(h, 0, n, ta.data_ptr(), n, info.data_ptr(), count))

    def potrs():
        check(lib.aclsolverSpotrsBatched(h, 0, n, nrhs, ta.data_ptr(), n, tb.data_ptr(), n, sinfo.data_ptr(), count))

    def both():
        potrf()
        potrs()

    def restore():
        A.copy_(A0)
        B.copy_(B0)

    steps = max(5, args.steps)
    for _ in range(3):
        timer(both, 1, restore)
    ms = timer(both, steps, restore)
    assert int(info.abs().max()) == 0 and int(sinfo[0].item()) == 0
    x = B.cpu().numpy().reshape(count, nrhs, n).transpose(0, 2, 1)
    ms_f = timer(potrf, steps, restore)
    ms_s = timer(potrs, steps, lambda: B.copy_(B0))
    # accuracy: normwise backward error of every solution in FP64
    r = b.astype(np.float64) - np.matmul(a.astype(np.float64), x.astype(np.float64))
    be = np.abs(r).max(axis=(1, 2)) / (np.abs(a).sum(axis=2).max(axis=1) * np.abs(x).max(axis=(1, 2))
                                       + np.abs(b).max(axis=(1, 2)))
    tri = n * (n + 1) // 2 * 4
    bytes_f, bytes_s = 2 * tri, tri + 2 * n * nrhs * 4
    flops_f, flops_s = n**3 / 3, 2 * n * n * nrhs

    cpu = None
    if args.cpu_seconds > 0:
        threads = host_lapack.max_threads()
        cpu_s, reps = cpu_timed(lambda: host_lapack.potrf_potrs(n, nrhs, a_cm, b_cm, count, threads=threads),
                                args.cpu_seconds)
        _, xc, ci = host_lapack.potrf_potrs(n, nrhs, a_cm, b_cm, count, threads=threads)
        xc = xc.reshape(count, nrhs, n).transpose(0, 2, 1)
        rc = b.astype(np.float64) - np.matmul(a.astype(np.float64), xc.astype(np.float64))
        bec = np.abs(rc).max(axis=(1, 2)) / (np.abs(a).sum(axis=2).max(axis=1) * np.abs(xc).max(axis=(1, 2))
                                             + np.abs(b).max(axis=(1, 2)))
        cpu = dict(host_lapack.describe(threads), value=round(count / cpu_s, 1), unit="solves/s", kind="openblas",
                   berr_max=float(bec.max()), info_max=int(ci.max()),
                   sample=f"all {count} matrices per pass (spotrf + spotrs, FP32 LAPACKE), {reps} passes")
    return {
        "workload": "10,000 SPD 32x32 (A = G G^T/32 + I), lower, lda 32, 1 RHS: SpotrfBatched + SpotrsBatched, fp32",
        "value": round(count / (ms * 1e-3), 1), "unit": "solves/s", "ms": round(ms, 5),
        "gflops": round(count * (flops_f + flops_s) / (ms * 1e-3) / 1e9, 1),
        "berr_max": float(be.max()),
        "roofline": roofline(count * (bytes_f + bytes_s), count * (flops_f + flops_s), ms,
                             "potrf_group_kernel<32,16> + solve_slot_check_kernel + potrs_lane_kernel<32>", "c1_potrf_potrs"),
        "kernels": {
            "potrf": roofline(count * bytes_f, count * flops_f, ms_f, "potrf_group_kernel<32,16>", "c1_potrf"),
            "potrs": roofline(count * bytes_s, count * flops_s, ms_s, "potrs_lane_kernel<32>", "c1_potrs"),
        },
        "l2": "inputs restored from a pristine copy, then a 256 MiB buffer written, before each step",
        "cpu_baseline": cpu,
    }


def measure_c2(handle, timer, args):
    """4,096 matrices of order 64 with N(0,1) entries (seed 1), one N(0,1) right-hand side:
    SgetrfBatched + SgetrsBatched + SgetriBatched (inverse out of place)."""
    import numpy as np
    import torch

    import aclsolver
    from oracle import host_lapack

    lib, check = aclsolver.library(), aclsolver.check
    count, n, nrhs = 4096, 64, 1
    rng = np.random.default_rng(1)
    a = rng.standard_normal((count, n, n), dtype=np.float32)
    b = rng.standard_normal((count, n, nrhs), dtype=np.float32)
    a_cm, b_cm = colmajor(a).reshape(-1), colmajor(b).reshape(-1)
    A0 = torch.from_numpy(a_cm).cuda()
    B0 = torch.from_numpy(b_cm).cuda()
    A, B, Cinv = torch.empty_like(A0), torch.empty_like(B0), torch.empty_like(A0)
    ta, tb = aclsolver.pointer_table(A, count, n * n * 4), aclsolver.pointer_table(B, count, n * nrhs * 4)
    tc = aclsolver.pointer_table(Cinv, count, n * n * 4)
    piv = torch.empty(count * n, dtype=torch.int32, device="cuda")
    info = torch.empty(count, dtype=torch.int32, device="cuda")
    sinfo = torch.empty(count, dtype=torch.int32, device="cuda")  # SgetrsBatched: one entry per matrix
    iinfo = torch.empty(count, dtype=torch.int32, device="cuda")
    h = handle.value

    def getrf():
        check(lib.aclsolverSgetrfBatched(h, n, ta.data_ptr(), n, piv.data_ptr(), info.data_ptr(), count))

    def getrs():
        check(lib.aclsolverSgetrsBatched(h, 0, n, nrhs, ta.data_ptr(), n, piv.data_ptr(), tb.data_ptr(), n,
                                         sinfo.data_ptr(), count))

    def getri():
        check(lib.aclsolverSgetriBatched(h, n, ta.data_ptr(), n, piv.data_ptr(), tc.data_ptr(), n, iinfo.data_ptr(),
                                         count))

    def all3():
        getrf()
        getrs()
        getri()

    def restore():
        A.copy_(A0)
        B.copy_(B0)

    steps = max(5, args.steps)
    for _ in range(3):
        timer(all3, 1, restore)
    ms = timer(all3, steps, restore)
    assert int(info.abs().max()) == 0 and int(sinfo.abs().max()) == 0 and int(iinfo.abs().max()) == 0
    x = B.cpu().numpy().reshape(count, nrhs, n).transpose(0, 2, 1)
    inv = Cinv.cpu().numpy().reshape(count, n, n).transpose(0, 2, 1)
    gpu_piv = piv.cpu().numpy().reshape(count, n)
    ms_f = timer(getrf, steps, restore)
    ms_s = timer(getrs, steps, lambda: B.copy_(B0))
    ms_i = timer(getri, steps)
    a64 = a.astype(np.float64)
    r = b.astype(np.float64) - np.matmul(a64, x.astype(np.float64))
    anorm = np.abs(a64).sum(axis=2).max(axis=1)
    be = np.abs(r).max(axis=(1, 2)) / (anorm * np.abs(x).max(axis=(1, 2)) + np.abs(b).max(axis=(1, 2)))
    # inverse: ||A X - I||_inf / (||A||_inf ||X||_inf) per matrix
    ri = np.matmul(a64, inv.astype(np.float64)) - np.eye(n)
    be_inv = np.abs(ri).sum(axis=2).max(axis=1) / (anorm * np.abs(inv).sum(axis=2).max(axis=1))

    mat, piv_b, vec = n * n * 4, n * 4, n * nrhs * 4
    bytes_f, bytes_s, bytes_i = 2 * mat + piv_b, mat + piv_b + 2 * vec, 2 * mat + piv_b
    flops_f, flops_s, flops_i = 2 * n**3 / 3, 2 * n * n * nrhs, 4 * n**3 / 3
    total_b, total_f = count * (bytes_f + bytes_s + bytes_i), count * (flops_f + flops_s + flops_i)

    cpu, cpiv = None, None
    if args.cpu_seconds > 0:
        threads = host_lapack.max_threads()
        cpu_s, reps = cpu_timed(lambda: host_lapack.getrf_getrs(n, nrhs, a_cm, b_cm, count, inverse=True,
                                                               threads=threads), args.cpu_seconds)
        _, _, _, cpiv, ci = host_lapack.getrf_getrs(n, nrhs, a_cm, b_cm, count, inverse=True, threads=threads)
        cpu = dict(host_lapack.describe(threads), value=round(count / cpu_s, 1),
                   unit="matrices/s (factor + solve + inverse)", kind="openblas", info_max=int(ci.max()),
                   sample=f"all {count} matrices per pass (sgetrf + sgetrs + sgetri, FP32 LAPACKE), {reps} passes")
    return {
        "workload": "4,096 N(0,1) 64x64, 1 RHS: SgetrfBatched + SgetrsBatched + SgetriBatched, fp32",
        "value": round(count / (ms * 1e-3), 1), "unit": "matrices/s (factor + solve + inverse)",
        "ms": round(ms, 5), "gflops": round(total_f / (ms * 1e-3) / 1e9, 1),
        "berr_max": float(be.max()), "inverse_residual_max": float(be_inv.max()),
        "ipiv_equal_openblas": None if cpiv is None else bool(np.array_equal(gpu_piv, cpiv.reshape(count, n))),
        "roofline": roofline(total_b, total_f, ms, "getrf_small_kernel<64> + getrs_small_kernel<64,0> + getri_small_kernel<64>",
                             "c2_all"),
        "kernels": {
            "getrf": roofline(count * bytes_f, count * flops_f, ms_f, "getrf_small_kernel<64>", "c2_getrf"),
            "getrs": roofline(count * bytes_s, count * flops_s, ms_s, "getrs_small_kernel<64,0>", "c2_getrs"),
            "getri": roofline(count * bytes_i, count * flops_i, ms_i, "getri_small_kernel<64>", "c2_getri"),
        },
        "l2": "inputs restored from a pristine copy, then a 256 MiB buffer written, before each step",
        "cpu_baseline": cpu,
    }


def make_c3_inputs(count=20_000, nrhs=4, seed=2):
    """Orders n_q ~ U{8..128}; A_q = G G^H / n + I with G's real and imaginary parts N(0,1);
    4 right-hand sides CN(0,1).  Returns flat column-major complex64 slabs (as float32) with
    per-matrix float offsets, lda = ldb = n."""
    import numpy as np

    rng = np.random.default_rng(seed)
    orders = rng.integers(8, 129, size=count).astype(np.int32)
    a_off = np.zeros(count, dtype=np.int64)
    b_off = np.zeros(count, dtype=np.int64)
    a_off[1:] = np.cumsum(2 * orders.astype(np.int64) ** 2)[:-1]
    b_off[1:] = np.cumsum(2 * orders.astype(np.int64) * nrhs)[:-1]
    a = np.empty(int(2 * (orders.astype(np.int64) ** 2).sum()), dtype=np.float32)
    b = rng.standard_normal(int(2 * orders.sum() * nrhs), dtype=np.float32) * np.float32(np.sqrt(0.5))
    for n in np.unique(orders):
        idx = np.nonzero(orders == n)[0]
        g = (rng.standard_normal((len(idx), n, n), dtype=np.float32)
             + 1j * rng.standard_normal((len(idx), n, n), dtype=np.float32)).astype(np.complex64)
        m = (np.matmul(g, np.conj(g.transpose(0, 2, 1))) / np.float32(n) + np.eye(n, dtype=np.complex64))
        m = m.astype(np.complex64)
        for k, q in enumerate(idx):
            # column-major: the transpose in C order, interleaved re/im
            a[a_off[q]:a_off[q] + 2 * n * n] = np.ascontiguousarray(m[k].T).view(np.float32).reshape(-1)
    return orders, a_off, b_off, a, b


def measure_c3(handle, timer, args):
    """20,000 HPD complex64 matrices of orders U{8..128}, 4 right-hand sides, one
    aclsolverCposvVbatched call (the persistent, size-bucketed, graph-captured launch)."""
    import ctypes as C

    import numpy as np
    import torch

    import aclsolver
    from oracle import host_lapack

    lib, check = aclsolver.library(), aclsolver.check
    count, nrhs = 20_000, 4
    orders, a_off, b_off, a, b = make_c3_inputs(count, nrhs)
    A0 = torch.from_numpy(a).cuda()
    B0 = torch.from_numpy(b).cuda()
    A, B = torch.empty_like(A0), torch.empty_like(B0)
    ta = torch.from_numpy(a_off * 4).cuda() + A.data_ptr()
    tb = torch.from_numpy(b_off * 4).cuda() + B.data_ptr()
    info = torch.empty(count, dtype=torch.int32, device="cuda")
    ld = np.ascontiguousarray(orders, dtype=np.int32)
    plan = C.c_void_p()
    t0 = time.perf_counter()
    check(lib.aclsolverCposvVbatchedPlanCreate(handle.value, 0, ld.ctypes.data, ld.ctypes.data, ld.ctypes.data, nrhs,
                                               count, 1, C.byref(plan)))
    plan_s = time.perf_counter() - t0

    def solve():
        check(lib.aclsolverCposvVbatched(handle.value, plan, ta.data_ptr(), tb.data_ptr(), info.data_ptr()))

    def restore():
        A.copy_(A0)
        B.copy_(B0)

    steps = max(5, args.steps // 2)
    for _ in range(3):
        timer(solve, 1, restore)
    ms = timer(solve, steps, restore)
    assert int(info.abs().max()) == 0
    xs = B.cpu().numpy()
    lib.aclsolverVbatchedPlanDestroy(plan)
    # backward error against FP64 on every 20th matrix
    be = []
    for q in range(0, count, 20):
        n = int(orders[q])
        m = a[a_off[q]:a_off[q] + 2 * n * n].view(np.complex64).reshape(n, n).T.astype(np.complex128)
        bq = b[b_off[q]:b_off[q] + 2 * n * nrhs].view(np.complex64).reshape(nrhs, n).T.astype(np.complex128)
        xq = xs[b_off[q]:b_off[q] + 2 * n * nrhs].view(np.complex64).reshape(nrhs, n).T.astype(np.complex128)
        r = bq - m @ xq
        be.append(np.abs(r).max() / (np.abs(m).sum(axis=1).max() * np.abs(xq).max() + np.abs(bq).max()))
    n64 = orders.astype(np.float64)
    tri = n64 * (n64 + 1) / 2 * 8
    total_b = float((3 * tri + 2 * n64 * nrhs * 8).sum())
    total_f = float((4 * n64**3 / 3 + 8 * n64**2 * nrhs).sum())

    cpu = None
    if args.cpu_seconds > 0:
        threads = host_lapack.max_threads()
        cpu_s, reps = cpu_timed(lambda: host_lapack.cpotrf_cpotrs_vbatched(orders, a_off, b_off, a, b, nrhs,
                                                                          threads=threads), args.cpu_seconds)
        _, _, ci = host_lapack.cpotrf_cpotrs_vbatched(orders, a_off, b_off, a, b, nrhs, threads=threads)
        cpu = dict(host_lapack.describe(threads), value=round(count / cpu_s, 1), unit="solves/s (4 RHS each)",
                   kind="openblas", info_max=int(ci.max()),
                   sample=f"all {count} matrices per pass (cpotrf + cpotrs, complex64 LAPACKE, dynamic chunks of "
                          f"4 matrices), {reps} passes")
    return {
        "workload": "20,000 HPD complex64, n ~ U{8..128}, A = G G^H/n + I, 4 RHS: one CposvVbatched call "
                    "(persistent, size-bucketed, graph-captured, autotuned)",
        "value": round(count / (ms * 1e-3), 1), "unit": "solves/s (4 RHS each)", "ms": round(ms, 5),
        "gflops": round(total_f / (ms * 1e-3) / 1e9, 1), "berr_max_sampled": float(max(be)),
        "berr_sample": f"every 20th matrix ({len(be)}), FP64",
        "plan_create_s": round(plan_s, 3),
        "roofline": roofline(total_b, total_f, ms, "vb_warp_kernel<32> + vb_cb_kernel<64> + vb_cb_kernel<128> (one graph)", "c3_vbatched"),
        "l2": "inputs (0.93 GB) restored from a pristine copy, then a 256 MiB buffer written, before each step",
        "cpu_baseline": cpu,
    }


# ---------------------------------------------------------------------------------------
# The single large system (config 5)
# ---------------------------------------------------------------------------------------

LARGE_N, LARGE_NRHS, LARGE_KAPPA = 8192, 16, 1e3


def measure_large(handle, args, steps=3):
    """The single large system beside the batched headline: one 8192 x 8192 A = U diag(s) V^T
    (Haar U, V from an FP64 QR on the GPU, kappa 1e3), 16 N(0,1) right-hand sides.  Plain:
    aclsolverSgetrf + aclsolverSgetrsBatched (FP32, the oracle's order) on device-resident
    copies; mixed: aclsolverSgesvIrBatched(BF16X3, tol 1e-7, maxIter 4).  Backward errors in
    FP64 on the GPU; forward errors against an FP64 LU solve (torch.linalg.solve)."""
    import ctypes as C
    import math

    import torch

    import aclsolver

    check = aclsolver.check
    lib = aclsolver.library()
    n, nrhs = LARGE_N, LARGE_NRHS
    g = torch.Generator(device="cuda").manual_seed(6)
    u, _ = torch.linalg.qr(torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g))
    v, _ = torch.linalg.qr(torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g))
    sv = torch.logspace(0.0, -math.log10(LARGE_KAPPA), n, device="cuda", dtype=torch.float64)
    a = ((u * sv) @ v.T).float()
    del u, v
    b = torch.randn(n, nrhs, device="cuda", generator=g)
    at, bt = a.T.contiguous(), b.T.contiguous()
    xt, work_a = torch.zeros_like(bt), torch.empty_like(at)
    ta, tb, tx, tw = (aclsolver.pointer_table(t, 1, 0) for t in (at, bt, xt, work_a))
    piv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    iters = torch.zeros(1, dtype=torch.int32, device="cuda")
    berr = torch.zeros(1, dtype=torch.float64, device="cuda")
    lw = C.c_int(0)
    check(lib.aclsolverSgetrf_bufferSize(handle.value, n, n, work_a.data_ptr(), n, C.byref(lw)))
    work = torch.empty(max(1, lw.value), device="cuda")
    stream = handle.stream

    def plain():
        check(lib.aclsolverSgetrf(handle.value, n, n, work_a.data_ptr(), n, work.data_ptr(), piv.data_ptr(),
                                  info.data_ptr()))
        check(lib.aclsolverSgetrsBatched(handle.value, 0, n, nrhs, tw.data_ptr(), n, piv.data_ptr(), tx.data_ptr(), n,
                                         info.data_ptr(), 1))

    def mixed():
        check(lib.aclsolverSgesvIrBatched(handle.value, aclsolver.FACTOR_BF16X3, n, nrhs, ta.data_ptr(), n,
                                          tb.data_ptr(), n, tx.data_ptr(), n, 4, 1e-7, iters.data_ptr(),
                                          berr.data_ptr(), info.data_ptr(), 1))

    def timed(fn, restore):
        best = []
        for _ in range(steps + 1):
            if restore:
                work_a.copy_(at)
                xt.copy_(bt)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            best.append(e0.elapsed_time(e1))
        rest = sorted(best[1:]) or best
        return rest[len(rest) // 2]  # median of the timed repetitions (after the first)

    a64, b64 = a.double(), b.double()
    x64 = torch.linalg.solve(a64, b64)
    anorm = a64.abs().sum(dim=1).max()

    def errors(x):
        x = x.double()
        r = b64 - a64 @ x
        be = r.abs().amax(dim=0) / (anorm * x.abs().amax(dim=0) + b64.abs().amax(dim=0))
        fe = (x - x64).abs().amax(dim=0) / x64.abs().amax(dim=0)
        return float(be.max()), float(fe.max())

    plain_ms = timed(plain, True)
    plain_be, plain_fe = errors(xt.T)
    mixed_ms = timed(mixed, False)
    mixed_be, mixed_fe = errors(xt.T)
    flops = 2.0 * n ** 3 / 3 + 2.0 * n * n * nrhs
    out = {
        "workload": f"one {n} x {n} system, A = U diag(s) V^T, kappa {LARGE_KAPPA:.0e}, {nrhs} right-hand sides",
        "plain": {"path": "Sgetrf + SgetrsBatched (FP32)", "ms": round(plain_ms, 3),
                  "gflops": round(flops / (plain_ms * 1e-3) / 1e9, 1), "berr_max": plain_be, "ferr_max": plain_fe},
        "mixed": {"path": "SgesvIrBatched(BF16X3, tol 1e-7, maxIter 4)", "ms": round(mixed_ms, 3),
                  "gflops": round(flops / (mixed_ms * 1e-3) / 1e9, 1), "berr_max": mixed_be, "ferr_max": mixed_fe,
                  "iterations": int(iters.item()), "berr_reported": float(berr.item())},
        "mixed_over_plain": round(plain_ms / mixed_ms, 3),
    }
    out["cholesky"] = measure_spotrf_large(handle, args)
    if args is not None and args.cpu_seconds > 0:
        from oracle import host_lapack

        threads = host_lapack.max_threads()
        a_h = at.cpu().numpy().reshape(-1)
        b_h = bt.cpu().numpy().reshape(-1)
        t0 = time.perf_counter()
        xc, st = host_lapack.sgesv(n, nrhs, a_h, b_h, threads=threads)
        dt = time.perf_counter() - t0
        be, fe = errors(torch.from_numpy(xc.reshape(nrhs, n)).cuda().T)
        out["cpu_baseline"] = dict(host_lapack.describe(threads), value=round(1.0 / dt, 3), unit="solves/s",
                                   ms=round(dt * 1e3, 1), kind="openblas", berr_max=be, ferr_max=fe, info=int(st),
                                   sample=f"one sgetrf + sgetrs ({nrhs} RHS, FP32 LAPACKE), OpenBLAS on {threads} threads")
    return out


def measure_spotrf_large(handle, args, n=4096, steps=3):
    """One 4096 x 4096 SPD matrix, A = G G^T / n + I (G ~ N(0,1) on the GPU, seed 7), lower:
    aclsolverSpotrf over the whole GPU (32-column panels, TMA-fed lower-triangle updates),
    device time of the call with the matrix restored before each repetition."""
    import torch

    import aclsolver

    lib = aclsolver.library()
    g = torch.Generator(device="cuda").manual_seed(7)
    G = torch.randn(n, n, device="cuda", generator=g)
    A0 = (G @ G.T / n + torch.eye(n, device="cuda")).contiguous()  # symmetric: its own column-major form
    del G
    A = torch.empty_like(A0)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = handle.stream
    times = []
    for _ in range(steps + 1):
        A.copy_(A0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        aclsolver.check(lib.aclsolverSpotrf(handle.value, 0, n, A.data_ptr(), n, None, 0, info.data_ptr()))
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    assert int(info.item()) == 0
    ms = sorted(times[1:])[len(times[1:]) // 2]
    # backward error of the factor: ||A - L L^T||_1 / ||A||_1 in FP64
    L = torch.triu(A).T.double()  # the column-major lower factor seen through torch's row-major view
    a64 = A0.double()
    rel = float((a64 - L @ L.T).abs().sum(dim=0).max() / a64.abs().sum(dim=0).max())
    out = {"workload": f"one {n} x {n} SPD matrix (G G^T / n + I), lower: aclsolverSpotrf",
           "ms": round(ms, 3), "gflops": round(n ** 3 / 3 / (ms * 1e-3) / 1e9, 1),
           "roofline": roofline(2.0 * n * (n + 1) / 2 * 4, n ** 3 / 3, ms, "potrf_syrk_kernel + diag + rows (per panel)"),
           "factor_residual": rel}
    if args is not None and args.cpu_seconds > 0:
        from oracle import host_lapack

        a_h = A0.cpu().numpy().reshape(-1)
        threads = host_lapack.max_threads()
        t0 = time.perf_counter()
        _, st = host_lapack.spotrf(n, a_h, threads=threads)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = dict(host_lapack.describe(threads), value=round(1.0 / dt, 3), unit="factorisations/s",
                                   ms=round(dt * 1e3, 1), kind="openblas", info=int(st),
                                   sample=f"one spotrf of the same matrix, OpenBLAS on {threads} threads")
    return out


def measure_complex_lu(handle, args, steps=3):
    """The complex LU family on its own workloads, device time per call (median of `steps`
    after one warm-up, inputs restored before each call):
      cgetrf   one 4096 x 4096 matrix of the reference's recipe (test/cgetrf/data/gen_data.py:
               integer real and imaginary parts 1..10), aclsolverCgetrf with pivots;
      cgetri   its inverse from the LU (aclsolverCgetri, the compensated column solves);
      cgetri_batched  10,000 LU factors of order 64 (aclsolverCgetriBatched);
      cmatinv  100,000 matrices of order 32 (aclsolverCmatinvBatched, Gauss-Jordan);
      cgetrs   one 4096 system with 64 right-hand sides through the host-buffer
               aclsolverCgetrs (row-major host A and B, copies inside the timed call)."""
    import numpy as np
    import torch

    import aclsolver

    lib = aclsolver.library()
    stream = handle.stream
    fp32 = fp32_peak_tflops()
    hbm, _, _ = peaks()

    def timed(call, restore=None):
        times = []
        for _ in range(steps + 1):
            if restore:
                restore()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        return sorted(times[1:])[len(times[1:]) // 2]

    out = {}
    n = 4096
    rng = np.random.RandomState(149)
    a_host = rng.randint(1, 11, size=(n, 2 * n)).astype(np.float32).view(np.complex64)
    a0 = torch.from_numpy(np.ascontiguousarray(a_host.T).view(np.float32).reshape(-1)).cuda()  # column-major
    a = torch.empty_like(a0)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    ms = timed(lambda: aclsolver.check(lib.aclsolverCgetrf(handle.value, n, n, a.data_ptr(), n, None,
                                                            ipiv.data_ptr(), info.data_ptr())),
               lambda: a.copy_(a0))
    assert int(info.item()) == 0
    flops = 8.0 * n ** 3 / 3
    out["cgetrf"] = {"workload": f"one {n} x {n} complex64 matrix (integer parts 1..10), partial pivoting",
                     "ms": round(ms, 3), "gflops": round(flops / (ms * 1e-3) / 1e9, 1),
                     "roofline": {"bound": "fp32 FMA (CUDA cores)", "achieved_tflops": round(flops / ms / 1e9, 2),
                                  "peak_tflops": fp32, "frac": round(flops / ms / 1e9 / fp32, 4)}}
    lu = a.clone()
    work = torch.empty(2 * n * n, dtype=torch.float32, device="cuda")
    inv = torch.empty_like(lu)
    ms = timed(lambda: aclsolver.check(lib.aclsolverCgetri(handle.value, n, inv.data_ptr(), n, ipiv.data_ptr(),
                                                            work.data_ptr(), n * n, info.data_ptr())),
               lambda: inv.copy_(lu))
    assert int(info.item()) == 0
    cflops = 36.0 * n ** 3  # n^3 compensated complex updates of 36 flops each
    out["cgetri"] = {"workload": f"inverse of that {n} x {n} LU in place (compensated column solves)",
                     "ms": round(ms, 3),
                     "roofline": {"bound": "fp32 (CUDA cores)", "achieved_tflops": round(cflops / ms / 1e9, 2),
                                  "peak_tflops": fp32, "frac": round(cflops / ms / 1e9 / fp32, 4)}}
    del work, inv

    # batched inverse from LU factors, order 64
    count, m = 10_000, 64
    g = torch.Generator(device="cuda").manual_seed(3)
    lus = torch.randn(count, m, m, 2, device="cuda", generator=g)
    lus[:, torch.arange(m), torch.arange(m), 0] += 2.0 * m  # a dominant diagonal keeps every factor regular
    lus = lus.reshape(-1).contiguous()
    piv = torch.arange(1, m + 1, dtype=torch.int32, device="cuda").repeat(count)
    outs = torch.empty_like(lus)
    tab_a = aclsolver.pointer_table(lus, count, m * m * 8)
    tab_c = aclsolver.pointer_table(outs, count, m * m * 8)
    infos = torch.zeros(count, dtype=torch.int32, device="cuda")
    ms = timed(lambda: aclsolver.check(lib.aclsolverCgetriBatched(handle.value, m, tab_a.data_ptr(), m, piv.data_ptr(),
                                                                   tab_c.data_ptr(), m, infos.data_ptr(), count)))
    assert int((infos != 0).sum().item()) == 0
    bytes_ = 2.0 * count * m * m * 8
    out["cgetri_batched"] = {"workload": f"{count:,} LU factors of order {m} (complex64), identity pivots",
                             "ms": round(ms, 3), "matrices_per_s": round(count / (ms * 1e-3), 1),
                             "roofline": {"bound": "fp32 (CUDA cores)",
                                          "achieved_tflops": round(36.0 * m ** 3 * count / ms / 1e9, 2),
                                          "peak_tflops": fp32, "hbm_gbs": round(bytes_ / ms / 1e6, 1),
                                          "hbm_frac": round(bytes_ / ms / 1e6 / hbm, 4)}}
    del lus, outs

    # direct inverse, order 32, the reference's inverse recipe
    count, m = 100_000, 32
    g = torch.Generator(device="cuda").manual_seed(4)
    mats = torch.randn(count, m, m, 2, device="cuda", generator=g)
    mats[:, torch.arange(m), torch.arange(m), :] += 4.0 * m ** 0.5
    mats = mats.reshape(-1).contiguous()
    outs = torch.empty_like(mats)
    tab_a = aclsolver.pointer_table(mats, count, m * m * 8)
    tab_c = aclsolver.pointer_table(outs, count, m * m * 8)
    infos = torch.zeros(count, dtype=torch.int32, device="cuda")
    ms = timed(lambda: aclsolver.check(lib.aclsolverCmatinvBatched(handle.value, m, tab_a.data_ptr(), m,
                                                                    tab_c.data_ptr(), m, infos.data_ptr(), count)))
    assert int((infos != 0).sum().item()) == 0
    bytes_ = 2.0 * count * m * m * 8
    gj = 8.0 * m ** 3 * count  # n^3 complex multiply-adds per Gauss-Jordan
    out["cmatinv"] = {"workload": f"{count:,} matrices of order {m} (complex64), Gauss-Jordan",
                      "ms": round(ms, 3), "matrices_per_s": round(count / (ms * 1e-3), 1),
                      "roofline": {"bound": "fp32 FMA (CUDA cores)", "achieved_tflops": round(gj / ms / 1e9, 2),
                                   "peak_tflops": fp32, "frac": round(gj / ms / 1e9 / fp32, 4),
                                   "hbm_gbs": round(bytes_ / ms / 1e6, 1), "hbm_frac": round(bytes_ / ms / 1e6 / hbm, 4)}}
    del mats, outs

    # host-buffer solve
    nrhs = 64
    lu_host = np.ascontiguousarray(lu.cpu().numpy().view(np.complex64).reshape(n, n).T)  # row-major LU
    piv_host = ipiv.cpu().numpy().astype(np.int32)
    b_host = (rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))).astype(np.complex64)
    hinfo = np.zeros(1, dtype=np.int32)
    times = []
    for _ in range(steps + 1):
        b = b_host.copy()
        t0 = time.perf_counter()
        st = lib.aclsolverCgetrs(handle.value, 0, n, nrhs, lu_host.ctypes.data, n, piv_host.ctypes.data,
                                 b.ctypes.data, nrhs, hinfo.ctypes.data)
        times.append((time.perf_counter() - t0) * 1e3)
        assert st == 0 and hinfo[0] == 0
    ms = sorted(times[1:])[len(times[1:]) // 2]
    out["cgetrs_host"] = {"workload": f"one {n} system, {nrhs} right-hand sides, host row-major buffers "
                                      "(H2D, layout, solve, D2H inside the call)",
                          "ms_wall": round(ms, 3), "h2d_bytes": n * n * 8 + n * nrhs * 8 + n * 4,
                          "d2h_bytes": n * nrhs * 8}
    if args is not None and args.cpu_seconds > 0:
        from scipy.linalg import lapack

        t0 = time.perf_counter()
        _, _, st = lapack.cgetrf(a_host)
        dt = time.perf_counter() - t0
        out["cgetrf"]["cpu_baseline"] = {"ms": round(dt * 1e3, 1), "kind": "scipy LAPACK cgetrf (OpenBLAS threads)",
                                         "info": int(st)}
    return out


def measure_qr(handle, args, steps=3):
    """The QR families: aclsolverSgeqrf of one 4096 x 4096 and one 2048 x 2048 N(0,1)
    matrix, aclsolverSSgels of a 4096 x 4096 system with one right-hand side, and their complex
    counterparts aclsolverCgeqrf / aclsolverCCgels at 4096 (device time per call, inputs
    restored before each).  `case_list_us` is the time the reference's own
    case lists carry for the same shape (test/sgeqrf/data/sgeqrf_cases.txt,
    test/sgels/data/sgels_cases.txt, a cuSOLVER run on the hardware those lists were made on)."""
    import ctypes as C

    import numpy as np
    import torch

    import aclsolver

    lib = aclsolver.library()
    stream = handle.stream
    fp32 = fp32_peak_tflops()

    def timed(call, restore):
        times = []
        for _ in range(steps + 1):
            restore()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        return sorted(times[1:])[len(times[1:]) // 2]

    out = {}
    g = torch.Generator(device="cuda").manual_seed(11)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    for n, listed in ((4096, 25449.6), (2048, 8781.9)):
        a0 = torch.randn(n * n, device="cuda", generator=g)
        a = torch.empty_like(a0)
        tau = torch.empty(n, device="cuda")
        work = torch.empty(2048, device="cuda")
        ms = timed(lambda: aclsolver.check(lib.aclsolverSgeqrf(handle.value, n, n, a.data_ptr(), n, tau.data_ptr(),
                                                                work.data_ptr(), 2048, info.data_ptr())),
                   lambda: a.copy_(a0))
        assert int(info.item()) == 0
        flops = 4.0 * n ** 3 / 3
        out[f"sgeqrf_{n}"] = {"workload": f"one {n} x {n} N(0,1) matrix: aclsolverSgeqrf", "ms": round(ms, 3),
                              "gflops": round(flops / (ms * 1e-3) / 1e9, 1),
                              "roofline": {"bound": "fp32 FMA (CUDA cores)", "frac": round(flops / ms / 1e9 / fp32, 4),
                                           "peak_tflops": fp32},
                              "case_list_us": listed}
        if n == 4096 and args is not None and args.cpu_seconds > 0:
            from scipy.linalg import lapack

            a_h = a0.cpu().numpy().reshape(n, n)
            t0 = time.perf_counter()
            lapack.sgeqrf(a_h)
            out[f"sgeqrf_{n}"]["cpu_baseline"] = {"ms": round((time.perf_counter() - t0) * 1e3, 1),
                                                  "kind": "scipy LAPACK sgeqrf (OpenBLAS threads)"}
    n = 4096
    a0 = torch.randn(n * n, device="cuda", generator=g)
    a = torch.empty_like(a0)
    b = torch.randn(n, device="cuda", generator=g)
    x = torch.empty(n, device="cuda")
    lw = C.c_size_t(0)
    aclsolver.check(lib.aclsolverSSgels_bufferSize(handle.value, n, n, 1, a.data_ptr(), n, b.data_ptr(), n,
                                                   x.data_ptr(), n, None, C.byref(lw)))
    work = torch.empty(lw.value // 4 + 1, device="cuda")
    niter = C.c_int(0)
    ms = timed(lambda: aclsolver.check(lib.aclsolverSSgels(handle.value, n, n, 1, a.data_ptr(), n, b.data_ptr(), n,
                                                           x.data_ptr(), n, work.data_ptr(), lw.value,
                                                           C.byref(niter), info.data_ptr())),
               lambda: a.copy_(a0))
    out["sgels_4096"] = {"workload": "4096 x 4096 system, 1 right-hand side: aclsolverSSgels", "ms": round(ms, 3),
                         "case_list_us": 30675.3}
    # complex family: Cgeqrf of one 4096 x 4096 matrix, CCgels of a 4096 x 4096 system (complex64,
    # real and imaginary parts N(0,1)); each call includes the reference's non-finite input screen
    a0 = torch.randn(2 * n * n, device="cuda", generator=g)
    a = torch.empty_like(a0)
    tau = torch.empty(2 * n, device="cuda")
    work = torch.empty(2 * 2048, device="cuda")
    ms = timed(lambda: aclsolver.check(lib.aclsolverCgeqrf(handle.value, n, n, a.data_ptr(), n, tau.data_ptr(),
                                                           work.data_ptr(), 2048, info.data_ptr())),
               lambda: a.copy_(a0))
    assert int(info.item()) == 0
    flops = 16.0 * n ** 3 / 3  # 4 n^3 / 3 complex multiply-adds, 4 real each
    out["cgeqrf_4096"] = {"workload": f"one {n} x {n} complex64 N(0,1) matrix: aclsolverCgeqrf", "ms": round(ms, 3),
                          "gflops": round(flops / (ms * 1e-3) / 1e9, 1),
                          "roofline": {"bound": "fp32 FMA (CUDA cores)", "frac": round(flops / ms / 1e9 / fp32, 4),
                                       "peak_tflops": fp32}}
    if args is not None and args.cpu_seconds > 0:
        from scipy.linalg import lapack

        a_h = a0.cpu().numpy().view(np.complex64).reshape(n, n)
        t0 = time.perf_counter()
        lapack.cgeqrf(a_h)
        out["cgeqrf_4096"]["cpu_baseline"] = {"ms": round((time.perf_counter() - t0) * 1e3, 1),
                                              "kind": "scipy LAPACK cgeqrf (OpenBLAS threads)"}
    b = torch.randn(2 * n, device="cuda", generator=g)
    x = torch.empty(2 * n, device="cuda")
    aclsolver.check(lib.aclsolverCCgels_bufferSize(handle.value, n, n, 1, a.data_ptr(), n, b.data_ptr(), n,
                                                   x.data_ptr(), n, None, C.byref(lw)))
    work = torch.empty(lw.value // 4 + 1, device="cuda")
    ms = timed(lambda: aclsolver.check(lib.aclsolverCCgels(handle.value, n, n, 1, a.data_ptr(), n, b.data_ptr(), n,
                                                           x.data_ptr(), n, work.data_ptr(), lw.value,
                                                           C.byref(niter), info.data_ptr())),
               lambda: a.copy_(a0))
    assert int(info.item()) == 0
    out["ccgels_4096"] = {"workload": "4096 x 4096 complex64 system, 1 right-hand side: aclsolverCCgels",
                          "ms": round(ms, 3)}
    return out


def run_profile_qr():
    """aclsolverSgeqrf of one 4096 x 4096 N(0,1) matrix, aclsolverSSgels of a 2048 x 2048
    system with 4 right-hand sides and aclsolverCgeqrf of one 2048 x 2048 complex64 matrix,
    once each, for an ncu capture."""
    import ctypes as C

    import torch

    import aclsolver

    lib = aclsolver.library()
    handle = aclsolver.Handle()
    g = torch.Generator(device="cuda").manual_seed(11)
    n = 4096
    a = torch.randn(n * n, device="cuda", generator=g)
    tau = torch.empty(n, device="cuda")
    work = torch.empty(2048, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    aclsolver.check(lib.aclsolverSgeqrf(handle.value, n, n, a.data_ptr(), n, tau.data_ptr(), work.data_ptr(), 2048,
                                        info.data_ptr()))
    n, r = 2048, 4
    a = torch.randn(n * n, device="cuda", generator=g)
    b = torch.randn(n * r, device="cuda", generator=g)
    x = torch.empty(n * r, device="cuda")
    lw = C.c_size_t(0)
    aclsolver.check(lib.aclsolverSSgels_bufferSize(handle.value, n, n, r, a.data_ptr(), n, b.data_ptr(), n,
                                                   x.data_ptr(), n, None, C.byref(lw)))
    ws = torch.empty(lw.value // 4 + 1, device="cuda")
    niter = C.c_int(0)
    aclsolver.check(lib.aclsolverSSgels(handle.value, n, n, r, a.data_ptr(), n, b.data_ptr(), n, x.data_ptr(), n,
                                        ws.data_ptr(), lw.value, C.byref(niter), info.data_ptr()))
    n = 2048
    a = torch.randn(2 * n * n, device="cuda", generator=g)
    tau = torch.empty(2 * n, device="cuda")
    work = torch.empty(2 * 2048, device="cuda")
    aclsolver.check(lib.aclsolverCgeqrf(handle.value, n, n, a.data_ptr(), n, tau.data_ptr(), work.data_ptr(), 2048,
                                        info.data_ptr()))
    torch.cuda.synchronize()
    handle.close()
    print("profile-qr done", flush=True)


def run_profile_complex():
    """Each complex LU workload once, for an ncu capture: Cgetrf of one 4096 x 4096 matrix
    (the reference recipe), CgetriBatched of 10,000 order-64 LU factors, CmatinvBatched of
    100,000 order-32 matrices, Cgetri of one 512 x 512 LU."""
    import numpy as np
    import torch

    import aclsolver

    lib = aclsolver.library()
    handle = aclsolver.Handle()
    n = 4096
    rng = np.random.RandomState(149)
    a_host = rng.randint(1, 11, size=(n, 2 * n)).astype(np.float32).view(np.complex64)
    a = torch.from_numpy(np.ascontiguousarray(a_host.T).view(np.float32).reshape(-1)).cuda()
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    aclsolver.check(lib.aclsolverCgetrf(handle.value, n, n, a.data_ptr(), n, None, ipiv.data_ptr(), info.data_ptr()))
    count, m = 10_000, 64
    g = torch.Generator(device="cuda").manual_seed(3)
    lus = torch.randn(count, m, m, 2, device="cuda", generator=g)
    lus[:, torch.arange(m), torch.arange(m), 0] += 2.0 * m
    lus = lus.reshape(-1).contiguous()
    piv = torch.arange(1, m + 1, dtype=torch.int32, device="cuda").repeat(count)
    outs = torch.empty_like(lus)
    infos = torch.zeros(count, dtype=torch.int32, device="cuda")
    tab_a, tab_c = aclsolver.pointer_table(lus, count, m * m * 8), aclsolver.pointer_table(outs, count, m * m * 8)
    aclsolver.check(lib.aclsolverCgetriBatched(handle.value, m, tab_a.data_ptr(), m, piv.data_ptr(), tab_c.data_ptr(),
                                               m, infos.data_ptr(), count))
    count, m = 100_000, 32
    mats = torch.randn(count, m, m, 2, device="cuda", generator=g)
    mats[:, torch.arange(m), torch.arange(m), :] += 4.0 * m ** 0.5
    mats = mats.reshape(-1).contiguous()
    outs = torch.empty_like(mats)
    infos = torch.zeros(count, dtype=torch.int32, device="cuda")
    tab_a, tab_c = aclsolver.pointer_table(mats, count, m * m * 8), aclsolver.pointer_table(outs, count, m * m * 8)
    aclsolver.check(lib.aclsolverCmatinvBatched(handle.value, m, tab_a.data_ptr(), m, tab_c.data_ptr(), m,
                                                infos.data_ptr(), count))
    m = 512
    sub = a.view(n, n, 2)[:m, :m].contiguous()  # a leading block of the LU: regular, identity pivots
    pv = torch.arange(1, m + 1, dtype=torch.int32, device="cuda")
    work = torch.empty(2 * m * m, dtype=torch.float32, device="cuda")
    aclsolver.check(lib.aclsolverCgetri(handle.value, m, sub.data_ptr(), m, pv.data_ptr(), work.data_ptr(), m * m,
                                        info.data_ptr()))
    torch.cuda.synchronize()
    handle.close()
    print("profile-complex done", flush=True)


# ---------------------------------------------------------------------------------------
# CPU baselines
# ---------------------------------------------------------------------------------------

def cpu_baseline_headline(args, a_cm, b_cm, x64):
    """The host LAPACK (OpenBLAS FP32 sgetrf + sgetrs) over all 256 systems of the headline
    workload, OpenMP over matrices, with the backward and forward errors of its solutions."""
    import numpy as np

    from oracle import host_lapack

    threads = host_lapack.max_threads()
    a_flat, b_flat = a_cm.reshape(-1), b_cm.reshape(-1)
    per_pass, reps = cpu_timed(lambda: host_lapack.getrf_getrs(N, NRHS, a_flat, b_flat, COUNT, threads=threads),
                               args.cpu_seconds)
    _, x, _, _, info = host_lapack.getrf_getrs(N, NRHS, a_flat, b_flat, COUNT, threads=threads)
    x = x.reshape(COUNT, NRHS, N).transpose(0, 2, 1)
    a = a_cm.transpose(0, 2, 1).astype(np.float64)
    b = b_cm.transpose(0, 2, 1).astype(np.float64)
    r = b - np.matmul(a, x.astype(np.float64))
    be = np.abs(r).max(axis=(1, 2)) / (np.abs(a).sum(axis=2).max(axis=1) * np.abs(x).max(axis=(1, 2))
                                       + np.abs(b).max(axis=(1, 2)))
    return dict(host_lapack.describe(threads), value=round(COUNT / per_pass, 2), unit=UNIT, kind="openblas",
                berr_max=float(be.max()), ferr_vs_fp64_max=float(forward_errors(x64, x).max()),
                info_max=int(info.max()),
                sample=f"all {COUNT} 512x512 systems per pass (sgetrf + sgetrs, FP32 LAPACKE, OpenMP over "
                       f"matrices, one OpenBLAS thread each), {reps} passes")


def run_reference(args, rank, world):
    """The reference's CPU path for this workload: the host FP32 LAPACK its tests use as the
    golden (OpenBLAS), over the same 256 systems, the same step count."""
    from oracle import host_lapack

    if rank != 0:
        return
    a, b = make_inputs(1)
    a_flat, b_flat = colmajor(a).reshape(-1), colmajor(b).reshape(-1)
    threads = host_lapack.max_threads()

    def step():
        host_lapack.getrf_getrs(N, NRHS, a_flat, b_flat, COUNT, threads=threads)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / max(1, args.steps)
    value = COUNT / dt
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 2),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(dt * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic: seeded U diag(s) V^T matrices and N(0,1) right-hand sides",
        "config": {"workload": WORKLOAD, "batch_per_gpu": COUNT, "n": N, "nrhs": NRHS, "kappa": list(KAPPAS),
                   "parallelism": f"replicas x{world}"},
        "cpu_baseline": dict(host_lapack.describe(threads), value=round(value, 2), unit=UNIT, kind="openblas",
                             sample=f"each step all {COUNT} 512x512 systems (sgetrf + sgetrs, FP32 LAPACKE, "
                                    "OpenMP over matrices, one OpenBLAS thread each)"),
        "e2e": {"value": round(value, 2), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# Profiling entry points (one launch of each hot kernel, for ncu)
# ---------------------------------------------------------------------------------------

def run_profile():
    """One launch of each hot kernel on the benchmark's inputs, for an ncu capture: the FP32
    and split-BF16 factorisations (aclsolverSgetrfBatchedMixed), the blocked solve
    (aclsolverSgetrsBatched) and one refinement call (maxIter 1)."""
    import torch

    import aclsolver

    lib = aclsolver.library()
    handle = aclsolver.Handle()
    a_host, b_host = make_inputs(1)
    a_cm, b_cm = colmajor(a_host), colmajor(b_host)
    A = torch.from_numpy(a_cm.reshape(-1)).cuda()
    B = torch.from_numpy(b_cm.reshape(-1)).cuda()
    W, X = torch.empty_like(A), torch.empty_like(B)
    ta, tb = aclsolver.pointer_table(A, COUNT, N * N * 4), aclsolver.pointer_table(B, COUNT, N * 4)
    tw, tx = aclsolver.pointer_table(W, COUNT, N * N * 4), aclsolver.pointer_table(X, COUNT, N * 4)
    piv = torch.zeros(COUNT * N, dtype=torch.int32, device="cuda")
    info = torch.zeros(COUNT, dtype=torch.int32, device="cuda")
    with torch.cuda.stream(handle.stream):
        for precision in (0, PRECISION):
            W.copy_(A)
            aclsolver.check(lib.aclsolverSgetrfBatchedMixed(handle.value, precision, N, tw.data_ptr(), N,
                                                            piv.data_ptr(), info.data_ptr(), COUNT))
        X.copy_(B)
        aclsolver.check(lib.aclsolverSgetrsBatched(handle.value, 0, N, NRHS, tw.data_ptr(), N, piv.data_ptr(),
                                                   tx.data_ptr(), N, info.data_ptr(), COUNT))
        aclsolver.check(lib.aclsolverSgesvIrBatched(handle.value, PRECISION, N, NRHS, ta.data_ptr(), N,
                                                    tb.data_ptr(), N, tx.data_ptr(), N, 1, TOL, None, None,
                                                    info.data_ptr(), COUNT))
    handle.stream.synchronize()
    print(json.dumps({"profile": "ok", "info_max": int(info.abs().max())}))
    handle.close()


def run_profile_small(args):
    """The plain batched workloads (configs 1-3) once each at full size, for an ncu launch
    list (`gpu__time_duration.sum` only), no CPU baselines."""
    import torch

    import aclsolver

    handle = aclsolver.Handle()
    aclsolver.check(aclsolver.library().aclsolverSetDeviceChecks(handle.value, 0))
    timer = DeviceTimer(handle.stream, torch.device("cuda"))
    args.cpu_seconds = 0.0
    args.steps = 1
    out = {}
    for key, fn in (("c1", measure_c1), ("c2", measure_c2), ("c3", measure_c3)):
        if key in args.profile_small:
            out[key] = fn(handle, timer, args)["ms"]
    print(json.dumps({"profile": "ok", "ms": out}))
    handle.close()


def run_profile_large():
    """The single large system for an ncu launch list: one plain factorisation and solve and
    one split-BF16 refinement call (the measurement of the 'large' key, one repetition)."""
    import aclsolver

    handle = aclsolver.Handle()
    out = measure_large(handle, None, steps=0)
    print(json.dumps({"profile": "ok", "large": out}))
    handle.close()


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(v, world):
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=3.0)
    ap.add_argument("--no-large", dest="large", action="store_false",
                    help="skip the single 8192 x 8192 system reported under the 'large' key")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="skip the plain batched workloads reported under the 'configs' key")
    ap.add_argument("--no-complex-lu", dest="complex_lu", action="store_false",
                    help="skip the complex LU and QR workloads reported under the 'complex_lu' and 'qr' keys")
    ap.add_argument("--profile-qr", action="store_true",
                    help="run Sgeqrf 4096 and SSgels 2048 once (for an ncu capture) and exit")
    ap.add_argument("--profile-complex", action="store_true",
                    help="run each complex LU workload once (for an ncu capture) and exit")
    ap.add_argument("--profile-large", action="store_true",
                    help="one large plain factorisation + solve and one large refinement call, for ncu")
    ap.add_argument("--profile", action="store_true",
                    help="run each hot kernel once on the workload (for an ncu capture) and exit")
    ap.add_argument("--profile-small", default="",
                    help="comma list of c1,c2,c3: run those plain batched workloads once (for ncu) and exit")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if args.impl == "b200":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl" if args.impl == "b200" else "gloo", timeout=datetime.timedelta(seconds=120))
    try:
        if args.profile:
            run_profile()
        elif args.profile_small:
            run_profile_small(args)
        elif args.profile_qr:
            run_profile_qr()
        elif args.profile_complex:
            run_profile_complex()
        elif args.profile_large:
            run_profile_large()
        elif args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_b200(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
