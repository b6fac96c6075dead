"""Benchmark: batched pivoted LU + solve + inverse on B200 through the aclsolver C ABI.

Workload (the reference's plain batched LU configuration): 4,096 matrices of order 64
with N(0,1) entries and one N(0,1) right-hand side each.  One step = the hot path over
the whole batch:
    aclsolverSgetrfBatched -> aclsolverSgetrsBatched -> aclsolverSgetriBatched
(P A = L U with the reference's pivot rule, x = A^-1 b, C = A^-1 from the factors).
`value` is solves/s with the inputs resident in HBM (device time, CUDA events on the
handle stream, summed over the K timed steps; before every step the input matrices are
restored from a pristine copy and a 256 MiB buffer is written so that no input is left
in the 126 MB L2).  `e2e` is the same step through the same C entry points with host
buffers: pinned host->device copy of A and b and device->host copy of x, A^-1, ipiv and
info inside the timed region.

`python bench.py --impl reference` times the reference's CPU path (the oracle, a C
restatement of the reference kernels' arithmetic) on this host with all its threads.

Multi-GPU (`torchrun ... bench.py --gpus N`): every rank runs its own batch of 4,096
matrices (the path is independent per matrix: replicas, no data-path collective); time
is the maximum over ranks and `value` the solves of all ranks over that time.
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

COUNT = 4096
N = 64
NRHS = 1
METRIC = "solves/s & GFLOP/s: mixed-prec+IR vs plain FP32, same B200, equal backward error"
UNIT = "solves/s"
WORKLOAD = "plain batched pivoted LU + solve + inverse, fp32, 4096 x 64x64, 1 RHS, N(0,1)"
# Algorithmic work per matrix (getrf 2n^3/3, getrs 2n^2 nrhs, getri 4n^3/3 flops; bytes:
# getrf reads and writes n^2 floats plus n pivots, getrs reads n^2 + pivots and reads and
# writes b, getri reads n^2 + pivots and writes n^2).
FLOPS = {"getrf": 2 * N**3 / 3, "getrs": 2 * N * N * NRHS, "getri": 4 * N**3 / 3}
BYTES = {
    "getrf": 2 * N * N * 4 + N * 4,
    "getrs": N * N * 4 + N * 4 + 2 * N * NRHS * 4,
    "getri": 2 * N * N * 4 + N * 4,
}
FALLBACK_HBM_GBS = 6650.0


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def traffic_summary():
    """Per-launch DRAM bytes of the dominant kernels from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            return {}
    return {}


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
                 "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
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


def make_inputs(seed):
    import numpy as np

    rng = np.random.default_rng(seed)
    a = rng.standard_normal((COUNT, N, N), dtype=np.float32)
    b = rng.standard_normal((COUNT, N, NRHS), dtype=np.float32)
    # column-major slabs: matrix q column j at q*N*N + j*N
    return np.ascontiguousarray(a.transpose(0, 2, 1)), np.ascontiguousarray(b.transpose(0, 2, 1))


def run_b200(args, rank, world):
    import numpy as np
    import torch

    import aclsolver

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    dev = torch.device("cuda", torch.cuda.current_device())
    lib = aclsolver.library()
    handle = aclsolver.Handle()
    aclsolver.check(lib.aclsolverSetDeviceChecks(handle.value, 0))
    stream = handle.stream

    a_host, b_host = make_inputs(1 + rank)
    a0 = torch.from_numpy(a_host.reshape(-1)).to(dev)
    b0 = torch.from_numpy(b_host.reshape(-1)).to(dev)
    a = torch.empty_like(a0)
    x = torch.empty_like(b0)
    c = torch.empty_like(a0)
    piv = torch.empty(COUNT * N, dtype=torch.int32, device=dev)
    info_f = torch.empty(COUNT, dtype=torch.int32, device=dev)
    info_s = torch.empty(COUNT, dtype=torch.int32, device=dev)
    info_i = torch.empty(COUNT, dtype=torch.int32, device=dev)
    ta = aclsolver.pointer_table(a, COUNT, N * N * 4)
    tx = aclsolver.pointer_table(x, COUNT, N * NRHS * 4)
    tc = aclsolver.pointer_table(c, COUNT, N * N * 4)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def solve():
        aclsolver.check(lib.aclsolverSgetrfBatched(handle.value, N, ta.data_ptr(), N, piv.data_ptr(),
                                                   info_f.data_ptr(), COUNT))
        ev[1].record(stream)
        aclsolver.check(lib.aclsolverSgetrsBatched(handle.value, 0, N, NRHS, ta.data_ptr(), N, piv.data_ptr(),
                                                   tx.data_ptr(), N, info_s.data_ptr(), COUNT))
        ev[2].record(stream)
        aclsolver.check(lib.aclsolverSgetriBatched(handle.value, N, ta.data_ptr(), N, piv.data_ptr(), tc.data_ptr(),
                                                   N, info_i.data_ptr(), COUNT))

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    totals = {"step": 0.0, "getrf": 0.0, "getrs": 0.0, "getri": 0.0}

    def step(timed):
        with torch.cuda.stream(stream):
            a.copy_(a0)
            x.copy_(b0)
            flush.fill_(timed & 0xFF)
            ev[0].record(stream)
            solve()
            ev[3].record(stream)
        if timed:
            ev[3].synchronize()
            totals["step"] += ev[0].elapsed_time(ev[3])
            totals["getrf"] += ev[0].elapsed_time(ev[1])
            totals["getrs"] += ev[1].elapsed_time(ev[2])
            totals["getri"] += ev[2].elapsed_time(ev[3])

    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()
    # correctness guard on the last warm-up output: every matrix factored and inverted
    assert int(info_f.abs().max()) == 0 and int(info_i.abs().max()) == 0, "unexpected info"

    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        wall0 = time.perf_counter()
        for i in range(args.steps):
            step(True if args.steps else False)
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
    barrier(world)
    ms = max_over_ranks(totals["step"] / args.steps, world)
    per_kernel = {k: totals[k] / args.steps for k in ("getrf", "getrs", "getri")}
    launches = 3  # one kernel per entry point with the device checks off

    # e2e: host buffers, copies inside the timed region
    a_pin = torch.from_numpy(a_host.reshape(-1)).pin_memory()
    b_pin = torch.from_numpy(b_host.reshape(-1)).pin_memory()
    x_pin = torch.empty(x.numel(), dtype=torch.float32).pin_memory()
    c_pin = torch.empty(c.numel(), dtype=torch.float32).pin_memory()
    p_pin = torch.empty(piv.numel(), dtype=torch.int32).pin_memory()
    i_pin = torch.empty(COUNT, dtype=torch.int32).pin_memory()
    e2e_steps = max(3, min(args.steps, 10))

    def e2e_step():
        with torch.cuda.stream(stream):
            a.copy_(a_pin, non_blocking=True)
            x.copy_(b_pin, non_blocking=True)
            solve()
            x_pin.copy_(x, non_blocking=True)
            c_pin.copy_(c, non_blocking=True)
            p_pin.copy_(piv, non_blocking=True)
            i_pin.copy_(info_i, non_blocking=True)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, world)
    assert bool(np.isfinite(x_pin.numpy()).all())
    h2d = COUNT * N * N * 4 + COUNT * N * NRHS * 4
    d2h = COUNT * N * NRHS * 4 + COUNT * N * N * 4 + COUNT * N * 4 + COUNT * 4

    if rank == 0:
        hbm, peak_kind = peaks()
        dominant = max(per_kernel, key=per_kernel.get)
        achieved = BYTES[dominant] * COUNT / (per_kernel[dominant] * 1e-3) / 1e9
        traffic = traffic_summary().get(dominant)
        total_flops = sum(FLOPS.values()) * COUNT * world
        value = COUNT * world / (ms * 1e-3)
        cpu = cpu_baseline(args)
        line = {
            "metric": METRIC,
            "value": round(value, 1),
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms, 5),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "fp32",
            "data": "synthetic: seeded N(0,1) matrices and right-hand sides",
            "config": {
                "workload": WORKLOAD,
                "batch_per_gpu": COUNT,
                "n": N,
                "nrhs": NRHS,
                "path": "SgetrfBatched + SgetrsBatched + SgetriBatched (device checks off)",
                "l2": "inputs restored from a pristine copy and a 256 MiB buffer written before each step",
                "parallelism": f"replicas x{world}",
            },
            "gflops": round(total_flops / (ms * 1e-3) / 1e9, 1),
            "per_kernel_ms": {k: round(v, 5) for k, v in per_kernel.items()},
            "roofline": {
                "kernel": dominant,
                "bound": "hbm",
                "achieved": round(achieved, 1),
                "peak": hbm,
                "peak_kind": peak_kind,
                "unit": "GB/s",
                "frac": round(achieved / hbm, 4),
                "traffic": traffic,
                "algorithmic_bytes_per_launch": BYTES[dominant] * COUNT,
                "step_hbm_frac": round(sum(BYTES.values()) * COUNT / (ms * 1e-3) / 1e9 / hbm, 4),
            },
            "e2e": {
                "value": round(COUNT * world / (e2e_ms * 1e-3), 1),
                "unit": UNIT,
                "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "ms_per_step": round(e2e_ms, 4),
            },
            "gpu_launches": launches * args.steps,
            "clocks": clocks.summary(),
            "wall_s_timed": round(wall, 4),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    handle.close()


def cpu_baseline(args):
    """The oracle (the reference's CPU path restated) on this host's cores."""
    import numpy as np

    import oracle

    a_host, b_host = make_inputs(1)
    a = np.ascontiguousarray(a_host.transpose(0, 2, 1))
    b = np.ascontiguousarray(b_host.transpose(0, 2, 1))
    threads = oracle.max_threads()
    reps, t0 = 0, time.perf_counter()
    while True:
        lu, ipiv, info = oracle.sgetrf_batched(a, threads=threads)
        oracle.sgetrs_batched(lu, ipiv, b, threads=threads)
        oracle.sgetri_batched(lu, ipiv, threads=threads)
        reps += 1
        if time.perf_counter() - t0 > args.cpu_seconds or reps >= 50:
            break
    dt = time.perf_counter() - t0
    return {
        "value": round(reps * COUNT / dt, 1),
        "unit": UNIT,
        "cores": threads,
        "kind": "port",
        "sample": f"{reps} passes of the full {COUNT} x {N}x{N} workload (getrf + getrs + getri), {dt:.1f} s",
    }


def run_reference(args, rank, world):
    import numpy as np

    import oracle

    if rank != 0:
        return
    a_host, b_host = make_inputs(1)
    a = np.ascontiguousarray(a_host.transpose(0, 2, 1))
    b = np.ascontiguousarray(b_host.transpose(0, 2, 1))
    threads = oracle.max_threads()

    def step():
        lu, ipiv, info = oracle.sgetrf_batched(a, threads=threads)
        oracle.sgetrs_batched(lu, ipiv, b, threads=threads)
        oracle.sgetri_batched(lu, ipiv, threads=threads)

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
        "value": round(value, 1),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(dt * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic: seeded N(0,1) matrices and right-hand sides",
        "config": {"workload": WORKLOAD, "batch_per_gpu": COUNT, "n": N, "nrhs": NRHS},
        "cpu_baseline": {
            "value": round(value, 1),
            "unit": UNIT,
            "cores": threads,
            "kind": "port",
            "sample": f"each step the full {COUNT} x {N}x{N} workload on the host (OpenMP over matrices)",
        },
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


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
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
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
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_b200(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
