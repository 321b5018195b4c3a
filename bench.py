#!/usr/bin/env python
"""Benchmark of the SpMV hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--dtype f64|f32]

Workload: CRS SpMV y = A*x on the irregular 2^22 x 2^22 matrix (row lengths
lognormal with mean 16 and sigma 1.0 clipped to [1, 4096], uniform unique
sorted columns, values U[-1,1], seed 1; 67,169,824 nonzeros), FP64 values and
int32 indices -- the configuration the headline HBM-bandwidth metric is quoted
on.  One step = one SpMV over the whole matrix.  The matrix (0.89 GB per step)
is far larger than L2 (126 MB), so no L2 flush is needed between steps.

Printed on rank 0 as one JSON line:
  value       device-resident throughput: algorithmic bytes of all ranks per
              step / max-over-ranks step time (CUDA events on the launching stream)
  e2e         the same metric through the C ABI's run() with pinned HOST x and y:
              H2D of x, the kernel, D2H of y and the synchronisation inside the
              timed region, every step
  roofline    the SpMV kernel against the measured HBM copy bandwidth
  cpu_baseline the reference's own OpenMP kernel (oracle/_ref) on the host cores
  clocks      nvidia-smi samples taken during the timed region

With N > 1 (torchrun) every rank owns one 2^22-row block of an N*2^22-square
matrix (weak scaling) and each step first all-gathers the distributed x with
NCCL, then runs the local SpMV: the exchange a row-distributed SpMV needs.

--impl reference times the reference's CPU implementation of the same SpMV
(oracle/_ref/libsmax_ref.so, all host threads) on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "SpMV/SpTRSV HBM GB/s (% of 8 TB/s); batched+adjoint vs plain on 1 B200 @1e-12"
UNIT = "GB/s"
N_ROWS = 1 << 22  # --rows overrides (a smaller case for profiling)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload: str):
    """Per-launch DRAM bytes of the SpMV kernel from the committed ncu summary."""
    p = os.path.join(REPO, "profiles", f"{workload}.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9]+)", open(p).read())
    return int(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_id_for_nvsmi(dev: int) -> str:
    import torch
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        return vis.split(",")[dev] if vis else str(dev)


def make_matrix(rank: int, world: int, vt):
    from smaxkernels_b200 import matrices as M
    n_cols = N_ROWS * world
    t0 = time.time()
    rp, col, val = M.lognormal_random(N_ROWS, seed=1 + rank, dtype=vt, n_cols=n_cols)
    log(f"[rank {rank}] matrix: n={N_ROWS} n_cols={n_cols} nnz={len(col)} ({time.time() - t0:.1f}s)")
    return rp, col, val


def cpu_reference_time(rp, col, val, x, max_s=20.0, reps=None):
    """Seconds per apply of the reference's OpenMP CRS SpMV on all host threads."""
    from oracle.oracle import Oracle, Reference, reference_available
    ncores = os.cpu_count() or 1
    if reference_available():
        R = Reference()
        threads = R.set_threads(ncores)
        t1, _ = R.time_spmv_crs(rp, col, val, x, warm=1, reps=1)
        n = reps or max(2, min(50, int(max_s / max(t1, 1e-6))))
        t, _ = R.time_spmv_crs(rp, col, val, x, warm=1, reps=n)
        return t, threads, "reference", n
    O = Oracle()
    t0 = time.perf_counter()
    O.spmv_crs(rp, col, val, x)
    t1 = time.perf_counter() - t0
    n = reps or max(1, min(20, int(max_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(n):
        O.spmv_crs(rp, col, val, x)
    return (time.perf_counter() - t0) / n, 1, "port", n


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    vt = np.float64 if args.dtype == "f64" else np.float32
    vbytes = np.dtype(vt).itemsize
    rp, col, val = make_matrix(0, 1, vt)
    x = np.random.default_rng(100).uniform(-1, 1, N_ROWS).astype(vt)
    from smaxkernels_b200.matrices import crs_bytes
    nbytes = crs_bytes(N_ROWS, len(col), N_ROWS, vbytes)
    budget = max(10.0, min(120.0, 0.5 * max(args.steps, 1)))
    t, threads, kind, n = cpu_reference_time(rp, col, val, x, max_s=budget)
    gbs = nbytes / t / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": round(gbs, 3), "unit": UNIT, "n_gpus": 0,
            "steps": n, "warmup": 1, "ms_per_step": round(t * 1e3, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.dtype,
            "data": "synthetic (seeded lognormal CRS matrix)",
            "config": config_dict(len(col), vbytes, 1),
            "cpu_baseline": {"value": round(gbs, 3), "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"{n} full applies of the workload after 1 warm-up"},
            "e2e": {"value": round(gbs, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def config_dict(nnz, vbytes, world):
    return {"workload": f"crs_spmv_{'f64' if vbytes == 8 else 'f32'}_lognormal_{N_ROWS}",
            "format": "CRS", "index": "int32", "n_rows_per_rank": N_ROWS, "n_cols": N_ROWS * world,
            "nnz_rank0": int(nnz), "row_length": "lognormal(mean 16, sigma 1.0), clip [1,4096]",
            "l2": "inputs larger than L2 (no flush)", "parallelism": f"row blocks x {world} ranks"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--rows", type=int, default=N_ROWS, help="rows per rank (default 2^22)")
    ap.add_argument("--variant", type=int, default=0, help="CRS kernel: 0 auto, 1 warp-stream, 2 row-tile")
    args = ap.parse_args()
    globals()["N_ROWS"] = args.rows
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from smaxkernels_b200 import FloatType, Interface, IntType, KernelType, PlatformType
    from smaxkernels_b200.matrices import crs_bytes

    vt = np.float64 if args.dtype == "f64" else np.float32
    tdt = torch.float64 if args.dtype == "f64" else torch.float32
    vbytes = np.dtype(vt).itemsize
    ft = FloatType.FLOAT64 if vbytes == 8 else FloatType.FLOAT32
    rp, col, val = make_matrix(rank, world, vt)
    nnz = len(col)
    n_cols = N_ROWS * world
    bytes_rank = crs_bytes(N_ROWS, nnz, n_cols, vbytes)

    # ---- device-resident path: x, y in HBM, the kernel on torch's stream ----
    smax = Interface()
    smax.register_kernel("spmv", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, ft)
    k = smax.kernel("spmv")
    if args.variant:
        k.set_spmv_variant(args.variant)
    x_local = torch.from_numpy(np.random.default_rng(100 + rank).uniform(-1, 1, N_ROWS).astype(vt)).cuda()
    x_glob = torch.empty(n_cols, dtype=tdt, device="cuda")
    y = torch.empty(N_ROWS, dtype=tdt, device="cuda")
    if world == 1:
        x_glob.copy_(x_local)
    k.register_A(N_ROWS, n_cols, nnz, col, rp, val)
    k.register_B(n_cols, x_glob)
    k.register_C(N_ROWS, y)
    # a dedicated stream: the kernels, the all-gather and the timing events
    # all run on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    k.set_stream(stream.cuda_stream)
    k.initialize()
    torch.cuda.synchronize()

    def step():
        if world > 1:
            dist.all_gather_into_tensor(x_glob, x_local)
        k.apply()

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_id_for_nvsmi(local)) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        t_dev = ev0.elapsed_time(ev1) * 1e-3 / args.steps
        if world > 1:
            tt = torch.tensor([t_dev], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t_dev = float(tt.item())

        # kernel-only time (no all-gather) for the roofline of the SpMV kernel
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            k.apply()
        ev1.record(stream)
        torch.cuda.synchronize()
        t_kernel = ev0.elapsed_time(ev1) * 1e-3 / args.steps

        # ---- end to end through the C ABI: pinned host x and y ----------------
        ke = None
        t_e2e = None
        if args.e2e_steps > 0:
            smax.register_kernel("spmv_host", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, ft)
            ke = smax.kernel("spmv_host")
            if args.variant:
                ke.set_spmv_variant(args.variant)
            xh = torch.empty(n_cols, dtype=tdt).pin_memory()
            yh = torch.empty(N_ROWS, dtype=tdt).pin_memory()
            xh.copy_(x_glob.cpu())
            ke.register_A(N_ROWS, n_cols, nnz, col, rp, val)
            ke.register_B(n_cols, xh.numpy())
            ke.register_C(N_ROWS, yh.numpy())
            ke.run()  # uploads A once; later runs move only x and y
            for _ in range(3):
                ke.run()
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            for _ in range(args.e2e_steps):
                ke.run()
            t_e2e = (time.perf_counter() - t0) / args.e2e_steps
            if world > 1:
                tt = torch.tensor([t_e2e], device="cuda", dtype=torch.float64)
                dist.all_reduce(tt, op=dist.ReduceOp.MAX)
                t_e2e = float(tt.item())
    clocks = clk.summary()

    # parity spot check of this run's output against the device result
    y_dev = y.cpu().numpy()
    if ke is not None:
        rel = float(np.linalg.norm(yh.numpy() - y_dev) / max(np.linalg.norm(y_dev), 1e-300))
        if rel > 1e-12:
            raise RuntimeError(f"host-path and device-path results differ: {rel}")

    total_bytes = bytes_rank * world
    if world > 1:
        tb = torch.tensor([float(bytes_rank)], device="cuda", dtype=torch.float64)
        dist.all_reduce(tb)
        total_bytes = float(tb.item())
    value = total_bytes / t_dev / 1e9

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t_cpu, threads, kind, n = cpu_reference_time(rp, col, val, x_glob.cpu().numpy(), max_s=20.0)
        cpu = {"value": round(bytes_rank / t_cpu / 1e9, 3), "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"{n} full applies of the same matrix (0.89 GB each) after 1 warm-up"}

    peak, peak_kind = measured_peaks()
    achieved = bytes_rank / t_kernel / 1e9
    workload = config_dict(nnz, vbytes, world)["workload"]
    traffic = ncu_traffic(workload)
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(t_dev * 1e3, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.dtype,
        "data": "synthetic (seeded lognormal CRS matrix, generated on the host)",
        "config": config_dict(nnz, vbytes, world),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} hbm_gbs",
                     "traffic": traffic, "algorithmic_bytes_per_launch": int(bytes_rank),
                     "kernel": "crs_tile_kernel" if args.variant == 2 else "crs_stream_kernel",
                     "kernel_ms": round(t_kernel * 1e3, 5)},
        "cpu_baseline": cpu,
        "e2e": None if t_e2e is None else {
            "value": round(bytes_rank * world / t_e2e / 1e9, 3), "unit": UNIT,
            "h2d_bytes_per_step": int(n_cols * vbytes), "d2h_bytes_per_step": int(N_ROWS * vbytes),
            "ms_per_step": round(t_e2e * 1e3, 4)},
        "gpu_launches": args.steps * (1 if args.variant == 2 else 2),  # SpMV kernel (+ carry fix-up) per step
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    smax.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
