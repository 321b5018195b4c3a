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


def cpu_reference_time(rp, col, val, x, max_s=20.0, reps=None, warm=1):
    """Seconds per apply of the reference's OpenMP CRS SpMV on all host threads
    (reps applies after warm warm-up applies; reps chosen to fill about max_s
    when not given)."""
    from oracle.oracle import Oracle, Reference, reference_available
    ncores = os.cpu_count() or 1
    if reference_available():
        R = Reference()
        threads = R.set_threads(ncores)
        t1, _ = R.time_spmv_crs(rp, col, val, x, warm=1, reps=1)
        n = reps or max(2, min(50, int(max_s / max(t1, 1e-6))))
        t, _ = R.time_spmv_crs(rp, col, val, x, warm=warm, reps=n)
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


def gather_floor_time(col, val, x_dev, n_cols, vt, stream, steps):
    """Seconds per pass of smax_measure_gather (L2-load gathers, two chunks in
    flight per warp) over this matrix's val/col, padded to 512-entry slices:
    the floor of the CRS SpMV's access pattern on this GPU."""
    import ctypes
    import torch
    from smaxkernels_b200 import _lib
    nnz = len(col)
    n_slices = (nnz + 511) // 512
    cd = torch.zeros(n_slices * 512, dtype=torch.int32, device="cuda")
    vd = torch.zeros(n_slices * 512, dtype=torch.float64 if vt == np.float64 else torch.float32, device="cuda")
    cd[:nnz] = torch.from_numpy(col).cuda()
    vd[:nnz] = torch.from_numpy(val).cuda()
    out = torch.empty(n_slices, dtype=vd.dtype, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    P = ctypes.c_void_p

    def probe():
        rc = _lib.lib.smax_measure_gather(1 if vt == np.float64 else 0, 0, 0, 2, n_slices, P(cd.data_ptr()),
                                          P(vd.data_ptr()), P(x_dev.data_ptr()), n_cols, P(out.data_ptr()),
                                          P(err.data_ptr()), P(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(_lib.lib.smax_last_error().decode())

    for _ in range(3):
        probe()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        probe()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) * 1e-3 / steps


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
    # one step = one full apply of the reference's OpenMP kernel (~16 ms on 16
    # host threads): exactly --steps applies after --warmup warm-up applies,
    # unless that would take longer than 4 minutes (the single-thread port)
    from oracle.oracle import reference_available
    steps, warm = max(args.steps, 1), max(args.warmup, 0)
    if not reference_available():
        steps = min(steps, 20)
    t, threads, kind, n = cpu_reference_time(rp, col, val, x, reps=steps, warm=warm)
    gbs = nbytes / t / 1e9
    # n_gpus: the launch's N (the reference runs on the host cores of rank 0)
    line = {"impl": "reference", "metric": METRIC, "value": round(gbs, 3), "unit": UNIT, "n_gpus": args.gpus,
            "steps": n, "warmup": warm, "ms_per_step": round(t * 1e3, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.dtype,
            "data": "synthetic (seeded lognormal CRS matrix)",
            "config": config_dict(len(col), vbytes, max(args.gpus, 1)),
            "cpu_baseline": {"value": round(gbs, 3), "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"{n} full applies of the workload after {warm} warm-up applies"
                                       + ("" if args.gpus <= 1 else
                                          " (the 2^22-row matrix of one rank: the per-rank block of the weak-scaled job)")},
            "e2e": {"value": round(gbs, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def config_dict(nnz, vbytes, world):
    return {"workload": f"crs_spmv_{'f64' if vbytes == 8 else 'f32'}_lognormal_{N_ROWS}",
            "format": "CRS", "index": "int32", "n_rows_per_rank": N_ROWS, "n_cols": N_ROWS * world,
            "nnz_rank0": int(nnz), "row_length": "lognormal(mean 16, sigma 1.0), clip [1,4096]",
            "l2": "inputs larger than L2 (no flush)", "parallelism": f"row blocks x {world} ranks"}


# ---------------------------------------------------------------------------
# The other workloads of the hot path (--workload NAME, or "all"): one JSON
# line per case, same keys as the headline line.  Single GPU.
# ---------------------------------------------------------------------------
EXTRA_WORKLOADS = ("gather_ceiling", "spmv_laplace64", "scs_spmv", "bcrs_spmv", "spmm", "spgemm", "sptrsv", "sptrsv_batch",
                   "sptrsv_refine", "adjoint", "solvers", "cusparse", "mtx", "colour")


class Bench:
    """Timing and reporting shared by the extra workloads."""

    def __init__(self, args):
        import torch
        self.torch = torch
        self.args = args
        self.stream = torch.cuda.Stream()
        torch.cuda.set_stream(self.stream)
        self.peak, self.peak_kind = measured_peaks()
        self.gpu = gpu_id_for_nvsmi(0)
        self._flush_buf = None
        self._flip = 0
        self.collect = None
        self.ref = None
        if not args.no_cpu_baseline:
            from oracle.oracle import Reference, reference_available
            if reference_available():
                self.ref = Reference()
                self.threads = self.ref.set_threads(os.cpu_count() or 1)

    # -- timing -----------------------------------------------------------
    def flush(self):
        """Writes 256 MB (twice the L2) so the next launch starts cold."""
        if self._flush_buf is None:
            self._flush_buf = self.torch.empty(256 << 20, dtype=self.torch.uint8, device="cuda")
        self._flip ^= 1
        self._flush_buf.fill_(self._flip)

    def time(self, fn, flush=False, budget_s=2.0, max_reps=None):
        """(seconds per call, calls timed): CUDA events on the bench stream,
        3 warm-up calls; with flush, each call is timed alone after an L2 flush."""
        torch = self.torch
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        fn()
        e1.record(self.stream)
        torch.cuda.synchronize()
        t1 = max(e0.elapsed_time(e1) * 1e-3, 1e-7)
        reps = int(min(max_reps or self.args.steps, max(3, budget_s / t1)))
        if not flush:
            e0.record(self.stream)
            for _ in range(reps):
                fn()
            e1.record(self.stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) * 1e-3 / reps, reps
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for a, b in evs:
            self.flush()
            a.record(self.stream)
            fn()
            b.record(self.stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs) * 1e-3 / reps, reps

    def clocks(self):
        return ClockSampler(self.gpu)

    # -- reporting --------------------------------------------------------
    def hbm(self, nbytes, t, kernel, workload=None):
        a = nbytes / t / 1e9
        return {"bound": "hbm", "achieved": round(a, 2), "peak": self.peak, "unit": "GB/s",
                "frac": round(a / self.peak, 4), "peak_source": f"{self.peak_kind} hbm_gbs",
                "traffic": ncu_traffic(workload) if workload else None,
                "algorithmic_bytes_per_launch": int(nbytes), "kernel": kernel}

    def cpu(self, timer, nbytes, sample, unit="GB/s"):
        if self.ref is None:
            return None
        t = timer()
        return {"value": round(nbytes / t / 1e9, 3), "unit": unit, "cores": self.threads, "kind": "reference",
                "sample": sample, "ms_per_call": round(t * 1e3, 4)}

    def emit(self, workload, metric, value, unit, t, reps, dtype, config, clocks, roofline=None, cpu=None,
             launches=None, higher=True, **extra):
        d = {"metric": metric, "value": round(value, 4), "unit": unit, "n_gpus": 1, "steps": reps, "warmup": 3,
             "ms_per_step": round(t * 1e3, 5), "higher_is_better": higher, "scaling": "weak", "vs_baseline": None,
             "dtype": dtype, "data": "synthetic (seeded, generated on the host)",
             "config": dict({"workload": workload}, **config), "roofline": roofline, "cpu_baseline": cpu,
             "e2e": None, "gpu_launches": launches, "clocks": clocks}
        d.update(extra)
        if self.collect is not None:  # gathered into the headline line instead of printed
            self.collect.append(d)
        else:
            print(json.dumps(d), flush=True)
        return d

    # -- kernels with device operands ---------------------------------------
    def kernel(self, ktype, vt, setup=None):
        from smaxkernels_b200 import FloatType, Interface, IntType, PlatformType
        smax = Interface()
        smax.register_kernel("k", ktype, PlatformType.CUDA, IntType.INT32,
                             FloatType.FLOAT64 if vt == np.float64 else FloatType.FLOAT32)
        k = smax.kernel("k")
        if setup:
            setup(k)
        return smax, k

    def dev(self, a):
        return self.torch.from_numpy(np.ascontiguousarray(a)).cuda()

    def zeros(self, n, vt):
        return self.torch.zeros(int(n), dtype=self.torch.float64 if vt == np.float64 else self.torch.float32,
                                device="cuda")


def _dt(vt):
    return "f64" if vt == np.float64 else "f32"


def wl_gather_ceiling(b: Bench):
    """The memory-traffic floor of the CRS SpMV on the lognormal 2^22 matrix
    (smax_measure_gather): val/col streamed exactly as the warp-stream kernel
    reads them and one x gather per entry, without row bookkeeping.  Lanes
    [0, tma_lanes) gather through TMA tile::gather4, the rest through L2 loads;
    the stream-only mode drops the gathers.  Every TMA configuration must give
    per-warp sums bit-identical to the all-L2-load one (same products, same
    order).  The CRS SpMV itself is timed on the same arrays for comparison."""
    import ctypes
    from smaxkernels_b200 import KernelType, _lib
    from smaxkernels_b200 import matrices as M
    from smaxkernels_b200.matrices import crs_bytes
    torch = b.torch
    dts = (np.float64, np.float32) if b.args.extra_dtype == "both" else \
        ((np.float64,) if b.args.extra_dtype == "f64" else (np.float32,))
    for vt in dts:
        vb = np.dtype(vt).itemsize
        rp, col, val = M.lognormal_random(1 << 22, seed=1, dtype=vt)
        n, nnz = len(rp) - 1, len(col)
        x = M.uniform_vector(n, 100, vt)
        n_slices = (nnz + 511) // 512
        colp = np.zeros(n_slices * 512, np.int32)
        colp[:nnz] = col
        valp = np.zeros(n_slices * 512, vt)
        valp[:nnz] = val
        cd, vd, xd = b.dev(colp), b.dev(valp), b.dev(x)
        out = b.zeros(n_slices, vt)
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        ft = 1 if vt == np.float64 else 0
        P = ctypes.c_void_p

        def probe(mode, lanes, depth):
            rc = _lib.lib.smax_measure_gather(ft, mode, lanes, depth, n_slices, P(cd.data_ptr()), P(vd.data_ptr()),
                                              P(xd.data_ptr()), n, P(out.data_ptr()), P(err.data_ptr()),
                                              P(b.stream.cuda_stream))
            if rc != 0:
                raise RuntimeError(_lib.lib.smax_last_error().decode())

        nbytes = crs_bytes(n, nnz, n, vb)
        stream_bytes = (vb + 4) * n_slices * 512
        results = {}
        with b.clocks() as clk:
            probe(0, 0, 2)
            torch.cuda.synchronize()
            ref_sums = out.clone()
            t, _ = b.time(lambda: probe(1, 0, 2))
            results["stream_only_d2"] = {"ms": round(t * 1e3, 5), "stream_gbs": round(stream_bytes / t / 1e9, 1)}
            for depth in (1, 2, 4):
                for lanes in (0, 8, 16, 24, 32):
                    out.fill_(0)
                    err.zero_()
                    probe(0, lanes, depth)
                    torch.cuda.synchronize()
                    same = bool(torch.equal(out, ref_sums)) and int(err.item()) == 0
                    t, _ = b.time(lambda: probe(0, lanes, depth))
                    results[f"tma{lanes}_d{depth}"] = {"ms": round(t * 1e3, 5),
                                                       "crs_equiv_gbs": round(nbytes / t / 1e9, 1),
                                                       "bit_identical": same}
            smax, k = b.kernel(KernelType.SPMV, vt)
            yd = b.zeros(n, vt)
            k.register_A(n, n, nnz, col, rp, val)
            k.register_B(n, xd)
            k.register_C(n, yd)
            k.set_stream(b.stream.cuda_stream)
            k.initialize()
            t_spmv, reps = b.time(k.apply)
            smax.close()
        best = min((v["ms"] for kk, v in results.items() if kk.startswith("tma")))
        b.emit(f"gather_ceiling_{_dt(vt)}_lognormal_4194304", "CRS SpMV traffic floor (ms per pass)", best, "ms",
               best * 1e-3, reps, _dt(vt),
               {"n_rows": n, "nnz": nnz, "n_slices": n_slices, "l2": "inputs larger than L2 (no flush)"},
               clk.summary(), b.hbm(nbytes, best * 1e-3, "gather_probe_kernel"), None, launches=reps, higher=False,
               probes=results, crs_spmv_ms=round(t_spmv * 1e3, 5),
               crs_spmv_frac_of_floor=round(best / (t_spmv * 1e3), 4))
        del cd, vd, xd, out
        torch.cuda.empty_cache()


def wl_spmv_laplace64(b: Bench):
    """CRS SpMV, 7-point 64^3 Laplacian (n = 262,144, nnz = 1,810,432): the
    27 MB working set is L2-resident, so report L2-flushed and hot."""
    from smaxkernels_b200 import KernelType
    from smaxkernels_b200 import matrices as M
    from smaxkernels_b200.matrices import crs_bytes
    rp, col, val = M.laplace3d_7pt(64)
    n, nnz = len(rp) - 1, len(col)
    x = M.uniform_vector(n, 0)
    smax, k = b.kernel(KernelType.SPMV, np.float64)
    xd, yd = b.dev(x), b.zeros(n, np.float64)
    k.register_A(n, n, nnz, col, rp, val)
    k.register_B(n, xd)
    k.register_C(n, yd)
    k.set_stream(b.stream.cuda_stream)
    k.initialize()
    nbytes = crs_bytes(n, nnz, n, 8)
    with b.clocks() as clk:
        t_fl, reps = b.time(k.apply, flush=True, budget_s=1.0, max_reps=200)
        t_hot, _ = b.time(k.apply)
        # the same without the per-apply CUDA-event stopwatch (SMAX_FLAG_TIMERS
        # = 0): at this size the event pair is a third of an apply
        k.set_timers(False)
        t_fl_off, _ = b.time(k.apply, flush=True, budget_s=1.0, max_reps=200)
        t_hot_off, _ = b.time(k.apply)
        k.set_timers(True)
    cpu = b.cpu(lambda: b.ref.time_spmv_crs(rp, col, val, x, warm=3, reps=100)[0], nbytes,
                "100 applies after 3 warm-ups (reference OpenMP CRS kernel)")
    b.emit("crs_spmv_f64_laplace3d_64", "CRS SpMV GB/s (L2-flushed)", nbytes / t_fl / 1e9, "GB/s", t_fl, reps,
           "f64", {"n_rows": n, "nnz": nnz, "l2": "flushed (256 MB write) before every timed launch"},
           clk.summary(), b.hbm(nbytes, t_fl, "crs_stream_kernel", "crs_spmv_f64_laplace3d_64"), cpu, launches=reps,
           hot={"value": round(nbytes / t_hot / 1e9, 3), "ms_per_step": round(t_hot * 1e3, 5),
                "l2": "hot (repeated launches, matrix L2-resident)"},
           timers_off={"value": round(nbytes / t_fl_off / 1e9, 3), "ms_per_step": round(t_fl_off * 1e3, 5),
                       "hot_value": round(nbytes / t_hot_off / 1e9, 3),
                       "hot_ms_per_step": round(t_hot_off * 1e3, 5)})
    smax.close()


def wl_scs_spmv(b: Bench):
    """SELL-32-1024 SpMV of the lognormal 2^22 matrix, FP64 and FP32."""
    from smaxkernels_b200 import KernelType
    from smaxkernels_b200 import matrices as M
    from smaxkernels_b200.matrices import crs_bytes
    dts = (np.float64, np.float32) if b.args.extra_dtype == "both" else \
        ((np.float64,) if b.args.extra_dtype == "f64" else (np.float32,))
    for vt in dts:
        vb = np.dtype(vt).itemsize
        rp, col, val = M.lognormal_random(1 << 22, seed=1, dtype=vt)
        n, nnz = len(rp) - 1, len(col)
        x = M.uniform_vector(n, 100, vt)
        smax, k = b.kernel(KernelType.SPMV, vt, lambda k: k.set_mat_scs(True))
        s = smax.utils.convert_crs_to_scs(n, n, nnz, col, rp, val, 32, 1024)
        vs = max(s["n_rows_padded"], n)
        xd = b.zeros(vs, vt)
        xd[:n] = b.dev(x)
        yd = b.zeros(vs, vt)
        k.register_A(32, 1024, s["n_rows"], s["n_rows_padded"], n, s["n_chunks"], s["n_elements"], s["nnz"],
                     s["chunk_ptr"], s["chunk_lengths"], s["col"], s["val"], s["perm"])
        k.register_B(vs, xd)
        k.register_C(vs, yd)
        k.set_stream(b.stream.cuda_stream)
        k.initialize()
        ne, nch, npad = s["n_elements"], s["n_chunks"], s["n_rows_padded"]
        # the kernel reads each row's entries up to its last non-padding one
        # (and one row length per padded row), not the layout's padding
        nbytes = (vb + 4) * nnz + 4 * npad + 4 * (nch + 1) + 4 * nch + vb * n + vb * npad
        stored = (vb + 4) * ne + 4 * (nch + 1) + 4 * nch + vb * n + vb * npad
        with b.clocks() as clk:
            t, reps = b.time(k.apply)
        cpu = b.cpu(lambda: b.ref.time_spmv_scs(s, x, warm=1, reps=20), nbytes,
                    "20 applies after 1 warm-up (reference OpenMP SELL-C-sigma kernel)")
        b.emit(f"scs_spmv_{_dt(vt)}_lognormal_4194304", "SELL-C-sigma SpMV GB/s (entries used, row lengths, x, y)",
               nbytes / t / 1e9, "GB/s", t, reps, _dt(vt),
               {"C": 32, "sigma": 1024, "n_rows": n, "nnz": nnz, "n_elements": ne,
                "l2": "inputs larger than L2 (no flush)"},
               clk.summary(), b.hbm(nbytes, t, "scs_task_kernel"), cpu, launches=reps,
               stored_bytes_gbs=round(stored / t / 1e9, 3),
               crs_equivalent_gbs=round(crs_bytes(n, nnz, n, vb) / t / 1e9, 3),
               gflops=round(2 * nnz / t / 1e9, 3))
        smax.close()
        del xd, yd
        b.torch.cuda.empty_cache()


def wl_bcrs_spmv(b: Bench):
    """4x4 BCRS SpMV of the lognormal 2^22 matrix, FP64 (n_blocks ~ nnz)."""
    from smaxkernels_b200 import KernelType
    from smaxkernels_b200 import matrices as M
    from smaxkernels_b200.matrices import crs_bytes
    vt, vb = np.float64, 8
    rp, col, val = M.lognormal_random(b.args.bcrs_rows, seed=1, dtype=vt)
    n, nnz = len(rp) - 1, len(col)
    x = M.uniform_vector(n, 100, vt)
    smax, k = b.kernel(KernelType.SPMV, vt, lambda k: k.set_mat_bcrs(True))
    bc = smax.utils.convert_crs_to_bcrs(n, n, nnz, col, rp, val, 4, 4, 4, 4, False)
    del rp, col, val
    xd, yd = b.dev(x), b.zeros(n, vt)
    k.register_A(bc["n_rows"], bc["n_cols"], bc["n_blocks"], 4, 4, 4, 4, bc["col"], bc["row_ptr"], bc["val"])
    k.register_B(n, xd)
    k.register_C(n, yd)
    k.set_stream(b.stream.cuda_stream)
    k.initialize()
    nb = bc["n_blocks"]
    nbytes = (16 * vb + 4) * nb + 4 * (bc["n_rows"] + 1) + vb * n + vb * n
    with b.clocks() as clk:
        t, reps = b.time(k.apply, budget_s=3.0)
    cpu = b.cpu(lambda: b.ref.time_spmv_bcrs(bc, x, False, warm=1, reps=5), nbytes,
                "5 applies after 1 warm-up (reference OpenMP BCRS kernel)")
    b.emit(f"bcrs4x4_spmv_f64_lognormal_{n}", "BCRS SpMV GB/s (stored bytes)", nbytes / t / 1e9, "GB/s", t,
           reps, "f64", {"block": "4x4", "n_blocks": nb, "nnz": nnz, "l2": "inputs larger than L2 (no flush)"},
           clk.summary(), b.hbm(nbytes, t, "bcrs_stream_kernel"), cpu, launches=reps,
           crs_equivalent_gbs=round(crs_bytes(n, nnz, n, vb) / t / 1e9, 3), gflops=round(2 * nnz / t / 1e9, 3))
    smax.close()


def wl_spmm(b: Bench):
    """Row-major SpMM with the 27-point 128^3 stencil (n = 2,097,152,
    nnz = 55,742,968), k = 16 and 64 vectors, FP64 and FP32."""
    from smaxkernels_b200 import KernelType
    from smaxkernels_b200 import matrices as M
    dts = (np.float64, np.float32) if b.args.extra_dtype == "both" else \
        ((np.float64,) if b.args.extra_dtype == "f64" else (np.float32,))
    ks = [int(v) for v in b.args.spmm_k.split(",")]
    variants = [int(v) for v in b.args.spmm_variants.split(",")]
    for vt in dts:
        vb = np.dtype(vt).itemsize
        rp, col, val = M.stencil27(128, dtype=vt)
        n, nnz = len(rp) - 1, len(col)
        for kv, var in [(kv, var) for kv in ks for var in variants]:
            X = np.random.default_rng(2).uniform(-1, 1, n * kv).astype(vt)
            smax, k = b.kernel(KernelType.SPMM, vt, lambda k: (k.set_vec_row_major(True), k.set_spmv_variant(var)))
            Xd, Yd = b.dev(X), b.zeros(n * kv, vt)
            k.register_A(n, n, nnz, col, rp, val)
            k.register_B(n, kv, Xd)
            k.register_C(n, kv, Yd)
            k.set_stream(b.stream.cuda_stream)
            k.initialize()
            nbytes = (vb + 4) * nnz + 4 * (n + 1) + 2 * vb * n * kv
            with b.clocks() as clk:
                t, reps = b.time(k.apply)
            cpu = b.cpu(lambda: b.ref.time_spmm(rp, col, val, X, kv, True, warm=1, reps=5), nbytes,
                        "5 applies after 1 warm-up (reference OpenMP row-major SpMM)") if var == variants[0] else None
            vname = {0: "", 1: "_grid", 2: "_walk"}[var]
            b.emit(f"spmm_rowmajor_k{kv}_{_dt(vt)}_stencil27_128{vname}", "SpMM GB/s", nbytes / t / 1e9, "GB/s", t,
                   reps, _dt(vt), {"n_rows": n, "nnz": nnz, "k": kv, "layout": "row-major X, Y",
                                   "l2": "inputs larger than L2 (no flush)",
                                   "kernel": "spmm_row_major_kernel" if var == 1 else "spmm_walk_kernel"},
                   clk.summary(), b.hbm(nbytes, t, "spmm_row_major_kernel" if var == 1 else "spmm_walk_kernel"),
                   cpu, launches=reps,
                   gflops=round(2 * nnz * kv / t / 1e9, 3))
            smax.close()
            del Xd, Yd
            b.torch.cuda.empty_cache()


def wl_spgemm(b: Bench):
    """C = A*A with the 7-point 96^3 Laplacian (n = 884,736, nnz(A) =
    6,137,856, nnz(C) = 21,732,480), FP64: symbolic + numeric per apply."""
    from smaxkernels_b200 import KernelType
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace3d_7pt(96)
    n, nnz = len(rp) - 1, len(col)
    smax, k = b.kernel(KernelType.SPGEMM, np.float64)
    k.register_A(n, n, nnz, col, rp, val)
    k.register_B(n, n, nnz, col, rp, val)
    k.register_C()
    k.set_stream(b.stream.cuda_stream)
    k.initialize()
    k.apply()
    k.finalize()
    c = k.result()
    nnz_c = int(c[2])
    lens = np.diff(rp)
    products = int(lens[col].sum())  # sum over A's entries of the length of B's row
    a_bytes = 12 * nnz + 4 * (n + 1)
    nbytes = 2 * a_bytes + 2 * a_bytes + 12 * nnz_c + 4 * (n + 1)
    # the kernel's phase timers (CUDA events): on the direct merge path
    # Fused_Gustavson is pass 1, Alloc_C the scan of C's counts and the
    # read-back of nnz(C), Compress the write pass
    phases = ("Symbolic_Setup", "Fused_Gustavson", "Alloc_C", "Compress")
    t0 = {nm: k.timer(nm) for nm in phases}
    with b.clocks() as clk:
        t, reps = b.time(k.apply, budget_s=2.0, max_reps=200)
    calls = reps + 4  # b.time's three warm-up calls and its first timed call
    phase_ms = {nm: round((k.timer(nm) - t0[nm]) / calls * 1e3, 4) for nm in phases}
    cpu = b.cpu(lambda: b.ref.time_spgemm(rp, col, val, reps=3), nbytes,
                "3 applies (reference OpenMP symbolic + numeric phases)")
    b.emit("spgemm_f64_laplace3d_96", "SpGEMM GB/s (2A + 2B + C bytes)", nbytes / t / 1e9, "GB/s", t, reps, "f64",
           {"n_rows": n, "nnz_a": nnz, "nnz_c": nnz_c, "products": products,
            "l2": "A, B (77 MB) L2-resident across the fused pass"},
           clk.summary(), b.hbm(nbytes, t, "gustavson_merge_write", "spgemm_f64_laplace3d_96"), cpu, launches=None,
           gflops=round(2 * products / t / 1e9, 3), reference_gflops_2nnzC=round(2 * nnz_c / t / 1e9, 3),
           phase_ms=phase_ms)
    smax.close()


def _tri_bytes(n, nnz, vb, kv=1):
    return (vb + 4) * nnz + 4 * (n + 1) + vb * n + 2 * vb * n * kv


def wl_sptrsv(b: Bench):
    """SpTRSV / SpTRSM, lower triangle of the 5-point 2048^2 Laplacian
    (n = 4,194,304, nnz = 12,578,816): natural order (4095 levels) in every
    launch scheme, the permuted level-scheduled flow, and k = 32 rows-major."""
    from smaxkernels_b200 import KernelType
    from smaxkernels_b200 import matrices as M
    vt, vb = np.float64, 8
    side = b.args.tri_side
    A = M.laplace2d_5pt(side)
    rp, col, val = M.lower_triangle(*A)
    n, nnz = len(rp) - 1, len(col)
    n_lv = 2 * side - 1
    rhs = M.uniform_vector(n, 3)
    names = {1: "per_level", 2: "merged", 3: "graph", 4: "persistent", 5: "syncfree"}
    results, xs = {}, {}
    cases = b.args.tri_cases.split(",")
    modes = [int(m) for m in b.args.tri_modes.split(",")] if "natural" in cases else []
    for mode in [m for m in (1, 2, 3, 4, 5) if m in modes]:
        smax, k = b.kernel(KernelType.SPTRSV, vt, lambda k: k.set_solve_mode(mode))
        xd, bd = b.zeros(n, vt), b.dev(rhs)
        k.register_A(n, n, nnz, col.copy(), rp, val.copy())
        k.register_B(n, xd)
        k.register_C(n, bd)
        k.set_stream(b.stream.cuda_stream)
        k.initialize()
        nbytes = _tri_bytes(n, nnz, vb)
        with b.clocks() as clk:
            t, reps = b.time(k.apply, budget_s=2.0, max_reps=100)
        results[mode] = t
        xs[mode] = xd.clone()
        same = bool(b.torch.equal(xd, xs[3])) if 3 in xs else None
        cpu = None
        if mode == 3:
            cpu = b.cpu(lambda: b.ref.time_sptrsv(rp, col, val, rhs, warm=1, reps=3)[0], nbytes,
                        "3 solves after 1 warm-up (reference naive_crs_sptrsv, serial)")
        b.emit(f"sptrsv_f64_laplace2d_{side}_natural_{names[mode]}", "SpTRSV GB/s", nbytes / t / 1e9, "GB/s", t,
               reps, "f64", {"n_rows": n, "nnz": nnz, "levels": n_lv, "scheme": names[mode]}, clk.summary(),
               b.hbm(nbytes, t, "syncfree_kernel" if mode == 5 else "wide_level_kernel/sweep_kernel"), cpu,
               launches=n_lv * reps if mode == 1 else (reps if mode == 4 else (2 * reps if mode == 5 else None)),
               us_per_level=round(t * 1e6 / n_lv, 4), bitwise_equal_to_graph=same)
        smax.close()
    if b.args.tri_natural_only:
        return
    if "permuted" in cases:
        # permuted flow: random symmetric permutation (seed 3), RS levels, level order
        Ar, Ac, Av, _ = M.random_symmetric_permutation(*A, seed=3)
        smax, k = b.kernel(KernelType.SPTRSV, vt)
        perm = np.zeros(n, np.int32)
        inv = np.zeros(n, np.int32)
        smax.utils.generate_perm(n, Ar, Ac, perm, inv, "RS")
        prp = np.zeros(n + 1, np.int32)
        pcol = np.zeros(len(Ac), np.int32)
        pval = np.zeros(len(Ac))
        smax.utils.apply_mat_perm(n, Ar, Ac, Av, prp, pcol, pval, perm, inv)
        lrp, lcol, lval = M.lower_triangle(prp, pcol, pval)
        lvl = np.array([smax.get_level_ptr_at(i) for i in range(smax.get_n_levels() + 1)], np.int32)
        nl = len(lvl) - 1
        xs = {}
        names[0] = "auto"
        for mode in [int(m) for m in b.args.tri_permuted_modes.split(",")]:
            smax.register_kernel(f"p{mode}", KernelType.SPTRSV, *b_types(vt))
            k = smax.kernel(f"p{mode}")
            k.set_mat_perm(True)
            k.set_solve_mode(mode)
            xd, bd = b.zeros(n, vt), b.dev(rhs)
            k.register_A(n, n, len(lcol), lcol.copy(), lrp, lval.copy())
            k.register_B(n, xd)
            k.register_C(n, bd)
            k.set_stream(b.stream.cuda_stream)
            k.initialize()
            nbytes = _tri_bytes(n, len(lcol), vb)
            with b.clocks() as clk:
                t, reps = b.time(k.apply, budget_s=2.0, max_reps=200)
            xs[mode] = xd.clone()
            same = bool(b.torch.equal(xs[mode], xs[3])) if 3 in xs else None
            cpu = None
            if mode == 3:
                cpu = b.cpu(lambda: b.ref.time_sptrsv(lrp, lcol, lval, rhs, levels=lvl, warm=1, reps=5)[0], nbytes,
                            "5 solves after 1 warm-up (reference crs_sptrsv_lvl, OpenMP within levels)")
            b.emit(f"sptrsv_f64_laplace2d_{side}_permuted_{names[mode]}", "SpTRSV GB/s", nbytes / t / 1e9, "GB/s", t,
                   reps, "f64", {"n_rows": n, "nnz": len(lcol), "levels": nl, "scheme": names[mode],
                                 "ordering": "random symmetric permutation (seed 3), RS level order"},
                   clk.summary(), b.hbm(nbytes, t, "syncfree_kernel" if mode in (0, 5) else "wide_level_kernel/sweep_kernel"),
                   cpu, launches=reps if mode == 4 else (2 * reps if mode in (0, 5) else None),
                   us_per_level=round(t * 1e6 / max(nl, 1), 4), bitwise_equal_to_graph=same)
        smax.close()
    if "sptrsm" in cases:
        # SpTRSM, k = 32 right-hand sides, row-major: graph-captured level
        # launches, then the default (the sync-free row kernel for this schedule)
        kv = 32
        B = np.random.default_rng(3).uniform(-1, 1, n * kv)
        xs_m = {}
        for mode in (3, 0):
            smax, k = b.kernel(KernelType.SPTRSM, vt, lambda k: (k.set_vec_row_major(True), k.set_solve_mode(mode)))
            Xd, Bd = b.zeros(n * kv, vt), b.dev(B)
            k.register_A(n, n, nnz, col.copy(), rp, val.copy())
            k.register_B(n, kv, Xd)
            k.register_C(n, kv, Bd)
            k.set_stream(b.stream.cuda_stream)
            k.initialize()
            nbytes = _tri_bytes(n, nnz, vb, kv)
            with b.clocks() as clk:
                t, reps = b.time(k.apply, budget_s=2.0, max_reps=50)
            xs_m[mode] = Xd.clone()
            same = bool(b.torch.equal(Xd, xs_m[3])) if mode != 3 else None
            cpu = b.cpu(lambda: b.ref.time_sptrsm(rp, col, val, B, kv, True, warm=0, reps=1), nbytes,
                        "1 solve (reference naive row-major SpTRSM, serial)") if mode == 3 else None
            tag = "graph" if mode == 3 else "auto"
            b.emit(f"sptrsm_k32_f64_laplace2d_{side}_natural_{tag}", "SpTRSM GB/s", nbytes / t / 1e9, "GB/s", t,
                   reps, "f64", {"n_rows": n, "nnz": nnz, "k": kv, "levels": n_lv, "layout": "row-major",
                                 "scheme": tag}, clk.summary(),
                   b.hbm(nbytes, t, "level_kernel/segment_kernel" if mode == 3 else "syncfree_rows_kernel"), cpu,
                   us_per_level=round(t * 1e6 / n_lv, 4), bitwise_equal_to_graph=same)
            smax.close()
            del Xd, Bd

def b_types(vt):
    from smaxkernels_b200 import FloatType, IntType, PlatformType
    return (PlatformType.CUDA, IntType.INT32, FloatType.FLOAT64 if vt == np.float64 else FloatType.FLOAT32)


def wl_sptrsv_batch(b: Bench):
    """64 lower triangles of 5-point Laplacians, sides 100 + round(600 i / 63):
    one persistent graph-captured launch vs one launch per level per matrix."""
    from smaxkernels_b200 import matrices as M
    from smaxkernels_b200.interface import TriangularBatch
    sides = [100 + int(round(600 * i / 63)) for i in range(64)]
    mats = [M.lower_triangle(*M.laplace2d_5pt(s)) for s in sides]
    tb = TriangularBatch(mats)
    n, total_levels, max_levels = tb.info()
    nnz = sum(len(m[1]) for m in mats)
    rhs = np.random.default_rng(3).uniform(-1, 1, n)
    bd, xd = b.dev(rhs), b.zeros(n, np.float64)
    nbytes = _tri_bytes(n, nnz, 8)
    times = {}
    names = {3: "persistent_graph", 2: "persistent", 1: "per_level"}
    # the per-level baseline first, so every line carries the speed-up over it
    for mode in (1, 3, 2):
        fn = lambda: tb.solve(bd, xd, mode, b.stream.cuda_stream)
        with b.clocks() as clk:
            t, reps = b.time(fn, budget_s=2.0, max_reps=200)
        times[mode] = t
        cpu = None
        if mode == 3 and b.ref is not None:
            def ref_time():
                return sum(b.ref.time_sptrsv(rp, c, v, np.ones(len(rp) - 1), warm=0, reps=1)[0]
                           for rp, c, v in mats)
            cpu = b.cpu(ref_time, nbytes, "1 solve of each of the 64 matrices (reference naive_crs_sptrsv)")
        b.emit(f"sptrsv_batch64_f64_laplace2d_{names[mode]}", "batched SpTRSV GB/s", nbytes / t / 1e9, "GB/s", t,
               reps, "f64", {"matrices": 64, "n_rows": n, "nnz": nnz, "total_levels": total_levels,
                             "max_levels": max_levels, "scheme": names[mode]}, clk.summary(),
               b.hbm(nbytes, t, "batch_sptrsv_kernel"), cpu,
               launches=total_levels * reps if mode == 1 else reps,
               speedup_vs_per_level=(round(times[1] / t, 3) if 1 in times else None))
    # the honest "why batch": the same 64 solves back to back, each a single
    # SpTRSV kernel with the platform's default (best) scheme for its matrix
    from smaxkernels_b200 import Interface, KernelType
    smax = Interface()
    ks = []
    for m, (rp, c, v) in enumerate(mats):
        nm = len(rp) - 1
        o = tb.row_offset(m)
        smax.register_kernel(f"t{m}", KernelType.SPTRSV)
        k = smax.kernel(f"t{m}")
        k.register_A(nm, nm, len(c), c.copy(), rp, v.copy())
        k.register_B(nm, xd[o:o + nm])
        k.register_C(nm, bd[o:o + nm])
        k.set_stream(b.stream.cuda_stream)
        k.initialize()
        ks.append(k)

    def singles():
        for k in ks:
            k.apply()
    with b.clocks() as clk:
        t1, reps = b.time(singles, budget_s=3.0, max_reps=50)
    b.emit("sptrsv_64_single_solves_f64_laplace2d", "64 single SpTRSV solves back to back (ms)", t1 * 1e3, "ms", t1,
           reps, "f64", {"matrices": 64, "n_rows": n, "nnz": nnz, "scheme": "one default SpTRSV kernel per matrix"},
           clk.summary(), b.hbm(nbytes, t1, "per-matrix solve kernels"), None, launches=None, higher=False,
           batch_speedup_over_singles=round(t1 / times[3], 3))
    smax.close()
    tb.close()


def wl_sptrsv_refine(b: Bench):
    """FP32 solve + FP64-residual refinement vs the FP64 solve, to 1e-12, on
    the 2048^2 lower triangle in natural order (4095 levels, latency-bound)
    and after the seed-3 random symmetric permutation with RS levels (15
    levels, bandwidth-side: where halving the value bytes could pay)."""
    from smaxkernels_b200 import Interface, KernelType
    from smaxkernels_b200 import matrices as M
    A = M.laplace2d_5pt(2048)
    n = len(A[0]) - 1
    rhs = M.uniform_vector(n, 3)
    bd = b.dev(rhs)
    cases = {"natural": (M.lower_triangle(*A), None)}
    Ar, Ac, Av, _ = M.random_symmetric_permutation(*A, seed=3)
    smax0 = Interface()
    perm = np.zeros(n, np.int32)
    inv = np.zeros(n, np.int32)
    smax0.utils.generate_perm(n, Ar, Ac, perm, inv, "RS")
    lvl = np.array([smax0.get_level_ptr_at(i) for i in range(smax0.get_n_levels() + 1)], np.int32)
    prp = np.zeros(n + 1, np.int32)
    pcol = np.zeros(len(Ac), np.int32)
    pval = np.zeros(len(Ac))
    smax0.utils.apply_mat_perm(n, Ar, Ac, Av, prp, pcol, pval, perm, inv)
    smax0.close()
    cases["permuted"] = (M.lower_triangle(prp, pcol, pval), lvl)
    for name, ((rp, col, val), levels) in cases.items():
        nnz = len(col)
        out = {}
        for steps in (0, 1, 2):
            def setup(k):
                k.set_refine(steps)
                if levels is not None:
                    k.set_mat_perm(True)
            smax, k = b.kernel(KernelType.SPTRSV, np.float64, setup)
            if levels is not None:
                smax.set_levels(levels)
            xd = b.zeros(n, np.float64)
            k.register_A(n, n, nnz, col.copy(), rp, val.copy())
            k.register_B(n, xd)
            k.register_C(n, bd)
            k.set_stream(b.stream.cuda_stream)
            k.initialize()
            with b.clocks() as clk:
                t, reps = b.time(k.apply, budget_s=2.0, max_reps=200)
            b.torch.cuda.synchronize()
            out[steps] = (t, reps, xd.clone(), clk.summary())
            smax.close()
        t64, _, x64, _ = out[0]
        errs = {s: float(b.torch.linalg.norm(out[s][2] - x64) / b.torch.linalg.norm(x64)) for s in (1, 2)}
        t32, reps, x32, clk = out[2]
        nbytes = _tri_bytes(n, nnz, 8)
        b.emit(f"sptrsv_refine2_vs_f64_laplace2d_2048_{name}", "refined FP32 SpTRSV speed-up over FP64",
               t64 / t32, "x", t32, reps, "f32+f64",
               {"n_rows": n, "nnz": nnz, "corrections": 2, "order": name,
                "levels": int(len(levels) - 1) if levels is not None else 4095}, clk,
               b.hbm(nbytes, t32, "solve kernels (FP32) + residual_kernel"), None,
               fp64_ms=round(t64 * 1e3, 4), refined1_ms=round(out[1][0] * 1e3, 4),
               refined2_ms=round(t32 * 1e3, 4), rel_diff_vs_fp64={"1": errs[1], "2": errs[2]})


def wl_adjoint(b: Bench):
    """Adjoint vs forward time: y = A x (7-point 64^3) and x = L^-1 b (lower
    5-point 512^2, 1023 levels), FP64; the adjoint computes d_in and d_val."""
    from smaxkernels_b200 import matrices as M
    from smaxkernels_b200.autograd import SparsePattern
    torch = b.torch
    cases = [("spmv_laplace3d_64", "spmv", M.laplace3d_7pt(64)),
             ("sptrsv_laplace2d_512", "sptrsv", M.lower_triangle(*M.laplace2d_5pt(512)))]
    for name, kind, (rp, col, val) in cases:
        n, nnz = len(rp) - 1, len(col)
        P = SparsePattern(rp, col, kind=kind)
        v = b.dev(val)
        xin = b.dev(M.uniform_vector(n, 4))
        P.forward(v, xin)
        xs = P._out.clone()  # the solve's x (or any x for SpMV)
        x_for_adj = xin if kind == "spmv" else xs
        P.k.set_stream(b.stream.cuda_stream)
        with b.clocks() as clk:
            tf, reps = b.time(P.k.apply, budget_s=1.0)
            ta, _ = b.time(lambda: P.k.adjoint(P._g, P._din, P._dval, x=x_for_adj), budget_s=1.0)
        b.emit(f"adjoint_{name}_f64", "adjoint time / forward time", ta / tf, "ratio", ta, reps, "f64",
               {"n_rows": n, "nnz": nnz, "outputs": "d_in and d_val"}, clk.summary(), None, None, higher=False,
               forward_ms=round(tf * 1e3, 5), adjoint_ms=round(ta * 1e3, 5))
        del P
        torch.cuda.empty_cache()


def _solver_iter_bytes(kind, n, nnz, nnz_u, nnz_l, vb, check_length):
    """Algorithmic bytes of one iteration (the residual every check_length
    iterations spread over them): each stored array and vector once."""
    resid = (vb + 4) * nnz + 4 * (n + 1) + 2 * vb * n
    if kind == "jacobi":  # A, x gathered once, D, b, x_new written
        it = (vb + 4) * nnz + 4 * (n + 1) + 4 * vb * n
    else:  # tmp = b - U x, then the D+L solve (b, x, D)
        it = (vb + 4) * nnz_u + 4 * (n + 1) + 3 * vb * n + _tri_bytes(n, nnz_l, vb)
    return it + resid / check_length


def wl_solvers(b: Bench):
    """The reference's Jacobi and Gauss-Seidel programs on device-resident
    operators: (1) the programs' own 10x10 Poisson problem to convergence,
    wall-clock time to solution for each driver next to the reference loop on
    the host; (2) the same operators on a 2048^2 grid, a fixed number of
    iterations (tol 0), per-iteration time and algorithmic GB/s."""
    import time as _time
    from smaxkernels_b200 import Interface
    from smaxkernels_b200 import matrices as M
    from smaxkernels_b200.solvers import Solver
    torch = b.torch
    st_ptr = b.stream.cuda_stream

    def problem(kind, nx):
        rp, col, val = M.poisson2d_app(nx)
        n = len(rp) - 1
        if kind == "jacobi":  # the program permutes A by BFS first (jacobi.cpp:82-91)
            smax = Interface()
            perm, inv = np.zeros(n, np.int32), np.zeros(n, np.int32)
            smax.utils.generate_perm(n, rp, col, perm, inv, "BFS")
            prp, pcol, pval = np.zeros(n + 1, np.int32), np.zeros(len(col), np.int32), np.zeros(len(col))
            smax.utils.apply_mat_perm(n, rp, col, val, prp, pcol, pval, perm, inv)
            smax.close()
            return prp, pcol, pval, np.ones(n), (np.ones(n) if kind == "jacobi" else np.zeros(n))
        return rp, col, val, np.ones(n), np.zeros(n)

    program_kinds = ("jacobi", "gauss_seidel") if b.args.solver_cases in ("all", "program") else ()
    for kind in program_kinds:
        rp, col, val, rhs, x0 = problem(kind, 10)
        n = len(rp) - 1
        bd, x0d = b.dev(rhs), b.dev(x0)
        xd = x0d.clone()
        res = {}
        with Solver(kind, rp, col, val) as s:
            for mode in ("device_loop", "graph_blocks", "plain"):
                def run():
                    xd.copy_(x0d)
                    return s.solve(bd, xd, mode=mode, stream=st_ptr)
                for _ in range(3):
                    run()
                ts = []
                for _ in range(30):
                    t0 = _time.perf_counter()
                    stt = run()
                    ts.append(_time.perf_counter() - t0)
                res[mode] = (float(np.median(ts)), stt)
        cpu = None
        if b.ref is not None:
            fn = b.ref.jacobi_app if kind == "jacobi" else b.ref.gauss_seidel_app
            tc = [fn(rp, col, val, rhs, x0)[4] for _ in range(20)]
            cpu = {"value": round(float(np.median(tc)) * 1e3, 5), "unit": "ms", "cores": b.threads,
                   "kind": "reference", "sample": "the program's loop through the reference's kernels, median of 20"}
        t, stt = res["device_loop"]
        b.emit(f"solver_{kind}_poisson2d_10_program", "time to solution (wall clock, host-synchronous call)",
               t * 1e3, "ms", t, 30, "f64", {"n_rows": n, "nnz": len(col), "tol": 1e-8, "check_length": 5,
                                            "driver": "device_loop"}, None, None, cpu, higher=False,
               n_iters=stt["n_iters"], residual=stt["residual_norm"],
               graph_blocks_ms=round(res["graph_blocks"][0] * 1e3, 4), plain_ms=round(res["plain"][0] * 1e3, 4))

    side = b.args.solver_side
    large_kinds = {"all": ("jacobi", "gauss_seidel", "gauss_seidel_pc"), "large": ("jacobi", "gauss_seidel",
                   "gauss_seidel_pc"), "large_jacobi": ("jacobi",)}.get(b.args.solver_cases, ())
    for kind in large_kinds:
        iters = b.args.solver_iters if kind != "gauss_seidel" else max(2, b.args.solver_iters // 20)
        if kind == "gauss_seidel_pc":
            # multicolour Gauss-Seidel: the matrix in PC colour order, so the
            # D+L solve has one level per colour
            rp0, col0, val0, _, _ = problem("gauss_seidel", side)
            n0 = len(rp0) - 1
            smax = Interface()
            perm, inv = np.zeros(n0, np.int32), np.zeros(n0, np.int32)
            smax.utils.generate_perm(n0, rp0, col0, perm, inv, "PC")
            rp, col, val = np.zeros(n0 + 1, np.int32), np.zeros(len(col0), np.int32), np.zeros(len(col0))
            smax.utils.apply_mat_perm(n0, rp0, col0, val0, rp, col, val, perm, inv)
            smax.close()
        else:
            rp, col, val, rhs, _ = problem(kind, side)
        n, nnz = len(rp) - 1, len(col)
        row_of = np.repeat(np.arange(n), np.diff(rp))
        nnz_l = int((col <= row_of).sum())
        nnz_u = nnz - nnz_l
        del row_of
        rhs = M.uniform_vector(n, 4)
        bd, x0d = b.dev(rhs), b.zeros(n, np.float64)
        xd = x0d.clone()
        cl = 5
        skind = "jacobi" if kind == "jacobi" else "gauss_seidel"
        with Solver(skind, rp, col, val) as s:
            def run():
                xd.copy_(x0d)
                s.solve(bd, xd, tol=0.0, max_iters=iters, check_length=cl, stream=st_ptr,
                        mode=b.args.solver_mode)
            with b.clocks() as clk:
                t, reps = b.time(run, budget_s=3.0, max_reps=20)
        t_it = t / iters
        nbytes = _solver_iter_bytes(skind, n, nnz, nnz_u, nnz_l, 8, cl)
        cpu = None
        if b.ref is not None:
            fn = b.ref.jacobi_app if kind == "jacobi" else b.ref.gauss_seidel_app
            k_cpu = 5 if kind == "jacobi" else 3
            tc = fn(rp, col, val, rhs, np.zeros(n), 0.0, k_cpu, cl)[4] / k_cpu
            cpu = {"value": round(nbytes / tc / 1e9, 3), "unit": "GB/s", "cores": b.threads, "kind": "reference",
                   "sample": f"{k_cpu} iterations of the program's loop through the reference's kernels",
                   "ms_per_iteration": round(tc * 1e3, 4)}
        kern = "jacobi_kernel" if kind == "jacobi" else "rhs_kernel + level-pack SpTRSV (sweep_kernel)"
        b.emit(f"solver_{kind}_poisson2d_{side}", "solver iteration GB/s (algorithmic bytes)", nbytes / t_it / 1e9,
               "GB/s", t_it, reps, "f64", {"n_rows": n, "nnz": nnz, "iterations": iters, "check_length": cl,
                                          "driver": b.args.solver_mode, "inputs": "larger than L2"},
               clk.summary(), b.hbm(nbytes, t_it, kern), cpu, ms_per_iteration=round(t_it * 1e3, 5))
        torch.cuda.empty_cache()


def wl_cusparse(b: Bench):
    """cuSPARSE, called through torch.sparse with the library's default
    algorithm choice, on the matrices of this platform's workloads (the
    reference's examples/benchmarks/cusparse_benchmarks measure the same
    operations: CSR SpMV, BSR SpMV, CSR SpMM).  One line per case: cuSPARSE's
    GB/s (the same algorithmic bytes as this platform's line), with this
    platform's time for the same operation on the same device arrays beside it."""
    from smaxkernels_b200 import KernelType
    from smaxkernels_b200 import matrices as M
    from smaxkernels_b200.matrices import crs_bytes
    torch = b.torch
    f64 = torch.float64

    def csr(rp, col, val, n_cols):
        return torch.sparse_csr_tensor(b.dev(rp.astype(np.int32)), b.dev(col.astype(np.int32)), b.dev(val),
                                       size=(len(rp) - 1, n_cols))

    def ours(k, **kw):
        """This platform's time per apply with its default stopwatches (a
        CUDA-event pair per apply), then with them off (SMAX_FLAG_TIMERS = 0),
        as torch.sparse records none."""
        t_on, _ = b.time(k.apply, **kw)
        k.set_timers(False)
        t_off, _ = b.time(k.apply, **kw)
        k.set_timers(True)
        return t_on, t_off

    def line(name, what, nbytes, t_lib, t_ours, reps, config, clk, kern_lib, extra=None):
        t_on, t_off = t_ours
        b.emit(name, f"cuSPARSE {what} GB/s (through torch.sparse)", nbytes / t_lib / 1e9, "GB/s", t_lib, reps,
               "f64", config, clk, b.hbm(nbytes, t_lib, kern_lib), None,
               ours_ms=round(t_on * 1e3, 5), cusparse_ms=round(t_lib * 1e3, 5),
               ours_over_cusparse=round(t_lib / t_on, 3), ours_ms_timers_off=round(t_off * 1e3, 5),
               ours_over_cusparse_timers_off=round(t_lib / t_off, 3), **(extra or {}))

    # CSR SpMV: the headline matrix and the 7-point 64^3 Laplacian
    for name, (rp, col, val), x in (
            ("lognormal_4194304", M.lognormal_random(1 << 22, seed=1), None),
            ("laplace3d_64", M.laplace3d_7pt(64), None)):
        n, nnz = len(rp) - 1, len(col)
        xd = b.dev(M.uniform_vector(n, 100))
        yd = b.zeros(n, np.float64)
        A = csr(rp, col, val, n)
        smax, k = b.kernel(KernelType.SPMV, np.float64)
        y2 = b.zeros(n, np.float64)
        k.register_A(n, n, nnz, col, rp, val)
        k.register_B(n, xd)
        k.register_C(n, y2)
        k.set_stream(b.stream.cuda_stream)
        k.initialize()
        with b.clocks() as clk:
            t_lib, reps = b.time(lambda: torch.mv(A, xd, out=yd))
            t_ours = ours(k)
        err = float(torch.linalg.norm(yd - y2) / torch.linalg.norm(y2))
        line(f"cusparse_csr_spmv_f64_{name}", "CSR SpMV", crs_bytes(n, nnz, n, 8), t_lib, t_ours, reps,
             {"n_rows": n, "nnz": nnz, "library_call": "torch.mv(sparse_csr, x)"}, clk.summary(),
             "cusparse SpMV (CSR)", {"rel_diff_vs_ours": err})
        smax.close()
        del A, xd, yd, y2
        torch.cuda.empty_cache()

    # CSR SpMM, 27-point 128^3, k = 16, row-major X
    rp, col, val = M.stencil27(128)
    n, nnz = len(rp) - 1, len(col)
    kv = 16
    X = b.dev(np.random.default_rng(2).uniform(-1, 1, n * kv))
    A = csr(rp, col, val, n)
    Y = torch.zeros(n, kv, dtype=f64, device="cuda")
    smax, k = b.kernel(KernelType.SPMM, np.float64, lambda k: k.set_vec_row_major(True))
    Y2 = b.zeros(n * kv, np.float64)
    k.register_A(n, n, nnz, col, rp, val)
    k.register_B(n, kv, X)
    k.register_C(n, kv, Y2)
    k.set_stream(b.stream.cuda_stream)
    k.initialize()
    X2 = X.view(n, kv)
    with b.clocks() as clk:
        t_lib, reps = b.time(lambda: torch.mm(A, X2, out=Y))
        t_ours = ours(k)
    err = float(torch.linalg.norm(Y.reshape(-1) - Y2) / torch.linalg.norm(Y2))
    line("cusparse_csr_spmm_k16_f64_stencil27_128", "CSR SpMM", (8 + 4) * nnz + 4 * (n + 1) + 2 * 8 * n * kv,
         t_lib, t_ours, reps, {"n_rows": n, "nnz": nnz, "k": kv, "library_call": "torch.mm(sparse_csr, X)"},
         clk.summary(), "cusparse SpMM (CSR)", {"rel_diff_vs_ours": err})
    smax.close()
    del A, X, Y, Y2, X2
    torch.cuda.empty_cache()

    # SpGEMM C = A*A, 7-point 96^3
    rp, col, val = M.laplace3d_7pt(96)
    n, nnz = len(rp) - 1, len(col)
    A = csr(rp, col, val, n)
    smax, k = b.kernel(KernelType.SPGEMM, np.float64)
    k.register_A(n, n, nnz, col, rp, val)
    k.register_B(n, n, nnz, col, rp, val)
    k.register_C()
    k.set_stream(b.stream.cuda_stream)
    k.initialize()
    k.apply()
    k.finalize()
    nnz_c = int(k.result()[2])
    a_bytes = 12 * nnz + 4 * (n + 1)
    nbytes = 4 * a_bytes + 12 * nnz_c + 4 * (n + 1)
    with b.clocks() as clk:
        t_lib, reps = b.time(lambda: torch.mm(A, A), budget_s=2.0, max_reps=100)
        t_ours = ours(k, budget_s=2.0, max_reps=100)
    C = torch.mm(A, A)
    line("cusparse_spgemm_f64_laplace3d_96", "SpGEMM", nbytes, t_lib, t_ours, reps,
         {"n_rows": n, "nnz_a": nnz, "nnz_c": nnz_c, "library_call": "torch.mm(sparse_csr, sparse_csr)"},
         clk.summary(), "cusparse SpGEMM", {"library_nnz_c": int(C._nnz())})
    smax.close()
    del A, C
    torch.cuda.empty_cache()

    # BSR 4x4 SpMV of the 7-point 64^3 Laplacian (the reference's harness uses
    # square blocks only)
    rp, col, val = M.laplace3d_7pt(64)
    n, nnz = len(rp) - 1, len(col)
    smax, k = b.kernel(KernelType.SPMV, np.float64, lambda k: k.set_mat_bcrs(True))
    bc = smax.utils.convert_crs_to_bcrs(n, n, nnz, col, rp, val, 4, 4, 4, 4, False)
    xd, yd, y2 = b.dev(M.uniform_vector(n, 100)), b.zeros(n, np.float64), b.zeros(n, np.float64)
    k.register_A(bc["n_rows"], bc["n_cols"], bc["n_blocks"], 4, 4, 4, 4, bc["col"], bc["row_ptr"], bc["val"])
    k.register_B(n, xd)
    k.register_C(n, y2)
    k.set_stream(b.stream.cuda_stream)
    k.initialize()
    nb = bc["n_blocks"]
    try:
        Ab = torch.sparse_bsr_tensor(b.dev(bc["row_ptr"]), b.dev(bc["col"]), b.dev(bc["val"]).view(nb, 4, 4),
                                     size=(n, n))
        with b.clocks() as clk:
            t_lib, reps = b.time(lambda: torch.mv(Ab, xd, out=yd))
            t_ours = ours(k)
        err = float(torch.linalg.norm(yd - y2) / torch.linalg.norm(y2))
        line("cusparse_bsr4x4_spmv_f64_laplace3d_64", "BSR SpMV", (16 * 8 + 4) * nb + 4 * (n // 4 + 1) + 16 * n,
             t_lib, t_ours, reps, {"n_rows": n, "n_blocks": nb, "library_call": "torch.mv(sparse_bsr, x)"},
             clk.summary(), "cusparse bsrmv", {"rel_diff_vs_ours": err})
    except RuntimeError as e:
        log(f"[bench] BSR SpMV through torch.sparse unavailable: {e}")
    smax.close()


def wl_mtx(b: Bench):
    """Matrix Market ingestion: the 7-point 64^3 Laplacian written as a
    coordinate file with its entries in scrambled order (1.8 M entries, full
    17-digit values), read back as CRS by this platform (threads parse
    line-aligned slices, the GPU sorts) and by the reference's own reader
    (examples/matrix_structs.hpp, fscanf) on the host."""
    import tempfile
    import time as _time
    from smaxkernels_b200 import Interface
    from smaxkernels_b200 import matrices as M
    rp, col, val = M.laplace3d_7pt(64)
    n, nnz = len(rp) - 1, len(col)
    row_of = np.repeat(np.arange(n), np.diff(rp))
    order = np.random.default_rng(7).permutation(nnz)
    vals = np.random.default_rng(8).uniform(-1, 1, nnz)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "laplace3d_64.mtx")
        with open(path, "w") as f:
            f.write("%%MatrixMarket matrix coordinate real general\n")
            f.write(f"{n} {n} {nnz}\n")
            np.savetxt(f, np.column_stack([row_of[order] + 1, col[order] + 1, vals[order]]),
                       fmt=["%d", "%d", "%.17g"])
        size = os.path.getsize(path)
        smax = Interface()
        smax.utils.read_mtx(path)  # warm-up (CUDA context, allocator)
        ts = []
        for _ in range(5):
            t0 = _time.perf_counter()
            got = smax.utils.read_mtx(path)
            ts.append(_time.perf_counter() - t0)
        t = float(np.median(ts))
        cpu = None
        if b.ref is not None:
            t0 = _time.perf_counter()
            ref = b.ref.read_mtx(path)
            tc = _time.perf_counter() - t0
            assert np.array_equal(ref[4], got[4]) and np.array_equal(ref[5], got[5])
            cpu = {"value": round(size / tc / 1e6, 3), "unit": "MB/s", "cores": 1, "kind": "reference",
                   "sample": "one read of the same file by the reference's reader (fscanf, one thread)",
                   "seconds": round(tc, 3)}
        b.emit("mtx_read_laplace3d_64", "Matrix Market ingestion MB/s (text bytes, wall clock)", size / t / 1e6,
               "MB/s", t, 5, "f64", {"n_rows": n, "nnz": nnz, "file_bytes": size, "parse_threads": os.cpu_count()},
               None, None, cpu, entries_per_s=round(nnz / t, 1))
        smax.close()


def wl_colour(b: Bench):
    """generate_perm with the colourings SC, PC and PC_BAL on the GPU: the
    5-point 2048^2 Laplacian (4.2 M rows, 2 colours) and the irregular
    lognormal 2^20 matrix; wall clock per call (host arrays in and out), next
    to the reference's generate_perm on one OpenMP thread (the setting in
    which its colourings are deterministic; the GPU result equals it)."""
    import time as _time
    from smaxkernels_b200 import Interface
    from smaxkernels_b200 import matrices as M
    cases = (("laplace2d_2048", lambda: M.laplace2d_5pt(2048)),
             ("lognormal_1048576", lambda: M.lognormal_random(1 << 20, seed=1)))
    for name, make in cases:
        rp, col, _ = make()
        n, nnz = len(rp) - 1, len(col)
        for t in ("SC", "PC", "PC_BAL"):
            smax = Interface()
            perm, inv = np.zeros(n, np.int32), np.zeros(n, np.int32)
            smax.utils.generate_perm(n, rp, col, perm, inv, t)  # warm-up
            ts = []
            for _ in range(3):
                t0 = _time.perf_counter()
                smax.utils.generate_perm(n, rp, col, perm, inv, t)
                ts.append(_time.perf_counter() - t0)
            n_col = smax.get_n_levels()
            smax.close()
            tg = float(np.median(ts))
            cpu = None
            if b.ref is not None:
                b.ref.set_threads(1)
                t0 = _time.perf_counter()
                rperm, _, rlvl = b.ref.generate_perm(rp, col, t)
                tc = _time.perf_counter() - t0
                b.ref.set_threads(os.cpu_count() or 1)
                same = bool(np.array_equal(rperm, perm) and len(rlvl) == n_col + 1)
                cpu = {"value": round(tc * 1e3, 3), "unit": "ms", "cores": 1, "kind": "reference",
                       "sample": "one generate_perm call of the reference on one OpenMP thread",
                       "identical_permutation": same}
            b.emit(f"colour_{t.lower()}_{name}", "generate_perm time (wall clock, host arrays)", tg * 1e3, "ms", tg,
                   3, "int32", {"n_rows": n, "nnz": nnz, "type": t}, None, None, cpu, higher=False,
                   n_colours=n_col)


ALSO_KEYS = ("value", "unit", "ms_per_step", "higher_is_better", "dtype", "us_per_level", "speedup_vs_per_level",
             "batch_speedup_over_singles", "bitwise_equal_to_graph")


def also_results(args):
    """The rest of the headline metric ("SpMV/SpTRSV ...; batched+adjoint vs
    plain"), measured in the same run on the same GPU: SpTRSV on the 2048^2
    lower triangle in natural order (default scheme: graph-captured level
    launches) and after the seed-3 permutation (default: sync-free), the
    64-matrix batch against one launch per level and against 64 single
    solves, and the SpMV / SpTRSV adjoints against their forward passes.
    Each entry is the compact form of that workload's own bench line."""
    import torch
    sub = argparse.Namespace(**vars(args))
    sub.tri_side, sub.tri_cases, sub.tri_modes, sub.tri_permuted_modes = 2048, "natural,permuted", "3", "0"
    sub.tri_natural_only = False
    b = Bench(sub)
    b.collect = []
    for fn in (wl_sptrsv, wl_sptrsv_batch, wl_adjoint):
        fn(b)
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    out = []
    for d in b.collect:
        e = {"workload": d["config"]["workload"], "metric": d["metric"]}
        e.update({k: d[k] for k in ALSO_KEYS if k in d and d[k] is not None})
        if d.get("roofline"):
            e["hbm_frac"] = d["roofline"]["frac"]
        if d.get("cpu_baseline"):
            e["cpu_baseline_ms"] = d["cpu_baseline"].get("ms_per_call")
        e["clocks"] = d.get("clocks")
        out.append(e)
    return out


def run_extra(args):
    import torch
    torch.cuda.set_device(0)
    b = Bench(args)
    names = EXTRA_WORKLOADS if args.workload == "all" else (args.workload,)
    for nm in names:
        log(f"[bench] workload {nm}")
        globals()[f"wl_{nm}"](b)
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--pipe-blocks", type=int, default=None,
                    help="e2e: row blocks of the host-pointer SpMV pipeline (default: the library's)")
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-also", action="store_true",
                    help="skip the SpTRSV / batch / adjoint companions of the headline line")
    ap.add_argument("--no-gather-floor", action="store_true",
                    help="skip the gather-floor measurement beside the headline kernel")
    ap.add_argument("--rows", type=int, default=N_ROWS, help="rows per rank (default 2^22)")
    ap.add_argument("--variant", type=int, default=0, help="CRS kernel: 0 auto, 1 warp-stream, 2 row-tile")
    ap.add_argument("--workload", default="crs_spmv", choices=("crs_spmv", "all") + EXTRA_WORKLOADS,
                    help="crs_spmv (the headline line) or another workload of the hot path (1 GPU)")
    ap.add_argument("--tri-side", type=int, default=2048, help="sptrsv workload: grid side of the Laplacian")
    ap.add_argument("--tri-modes", default="1,2,3,4,5", help="sptrsv workload: solve modes of the natural case")
    ap.add_argument("--tri-natural-only", action="store_true", help="sptrsv workload: natural order only")
    ap.add_argument("--tri-cases", default="natural,permuted,sptrsm",
                    help="sptrsv workload: cases to run (natural, permuted, sptrsm)")
    ap.add_argument("--tri-permuted-modes", default="3,0,4,5",
                    help="sptrsv workload: solve modes of the permuted case (0 = the default scheme)")
    ap.add_argument("--extra-dtype", default="both", choices=("both", "f64", "f32"),
                    help="scs_spmv / spmm workloads: value types to run")
    ap.add_argument("--spmm-k", default="16,64", help="spmm workload: vector counts")
    ap.add_argument("--spmm-variants", default="0",
                    help="spmm workload: row-major kernels (0 default, 1 all-rows grid, 2 per-SM row walks)")
    ap.add_argument("--bcrs-rows", type=int, default=1 << 22, help="bcrs_spmv workload: rows of the matrix")
    ap.add_argument("--solver-side", type=int, default=2048, help="solvers workload: grid side of the large case")
    ap.add_argument("--solver-cases", default="all", choices=("all", "program", "large", "large_jacobi"),
                    help="solvers workload: the programs' 10x10 problem, the large grid (or only its Jacobi case), "
                         "or both")
    ap.add_argument("--solver-mode", default="device_loop", choices=("device_loop", "graph_blocks", "plain"),
                    help="solvers workload: driver of the large-grid case")
    ap.add_argument("--solver-iters", type=int, default=200,
                    help="solvers workload: Jacobi iterations of the large case (Gauss-Seidel: 1/20 of it)")
    args = ap.parse_args()
    globals()["N_ROWS"] = args.rows
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "crs_spmv":
        return run_extra(args)

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
        t_floor = None if args.no_gather_floor else gather_floor_time(col, val, x_glob, n_cols, vt, stream,
                                                                      args.steps)

        # ---- end to end through the C ABI: pinned host x and y ----------------
        ke = None
        t_e2e = None
        if args.e2e_steps > 0:
            smax.register_kernel("spmv_host", KernelType.SPMV, PlatformType.CUDA, IntType.INT32, ft)
            ke = smax.kernel("spmv_host")
            if args.pipe_blocks is not None:
                ke.set_spmv_pipeline(args.pipe_blocks)
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
        # the host path's row blocks cut the entry slices elsewhere, so the
        # sums round differently: the parity tolerance of the value type
        if rel > (1e-12 if args.dtype == "f64" else 1e-5):
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

    also = None
    if world == 1 and not args.no_also:
        # outside every timed region above: each companion times itself
        also = also_results(args)
        torch.cuda.set_stream(stream)

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
        "gather_floor": None if t_floor is None else {
            "ms": round(t_floor * 1e3, 5), "frac_of_floor": round(t_floor / t_kernel, 4),
            "what": "smax_measure_gather on this rank's matrix: the same val/col stream and one x gather per "
                    "entry through L2 loads, no row bookkeeping (the request-rate floor of this access pattern)"},
        "also": also,
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
