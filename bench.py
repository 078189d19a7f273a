#!/usr/bin/env python
"""GSE-k reciprocal-space force evaluations per second on B200.

One step = one whole GSE-k force evaluation of a 262,143-charge water-like
box (L = 140 A, M = 144, sigma = 2, kappa = 0.4, lambda_sigma1 = 3):
spreadCharge1 -> solvePoisson -> calculateEnergy -> interpolateForce.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision mixed|fp64]

`value` is whole-job evals/s with inputs resident in HBM (CUDA events around
each evaluation; L2 is flushed between timed evaluations).  `e2e` is the same
metric through the public call with pinned host buffers (host->device copy of
the positions and device->host copy of forces and energy inside every step).
With N > 1 (torchrun) every rank evaluates its own independent replica:
replicas only, no collective on the data path.  The batched workload (256
independent systems) is partitioned across the ranks (gse_b200.multi) and
reported as 256 systems over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import datetime
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

METRIC = "GSE recip force evals/s at 262k charges: mixed vs FP64 GPU at ≤1e-4 rel force RMS"
UNIT = "force evals/s"
WORKLOAD = "water_262143_L140_M144"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

# algorithmic bytes per launch (262,143 charges, M = 144): positions+charges
# read once, grid written or read once, forces written once (float64)
N_ATOMS = 262143
GRID = 144 ** 3


def algorithmic_bytes(stage: str, precision: str) -> float:
    ct = 4 if precision == "mixed" else 8
    xyzq = N_ATOMS * 4 * ct
    grid = GRID * ct
    forces = N_ATOMS * 3 * 8
    if stage == "spread":
        return xyzq + grid
    if stage == "gather":
        return xyzq + grid + forces
    raise ValueError(stage)


# algorithmic flops per launch (262,143 charges, M = 144, stencil 13): the
# spread adds 2197 cube points per atom (multiply and add), the gather visits
# 704.5 points per atom inside the cut-off sphere on average (8 flops each:
# the weight, its products with the potential and the three offsets)
GATHER_POINTS_PER_ATOM = 704.5


def algorithmic_flops(stage: str) -> float:
    if stage == "spread":
        return N_ATOMS * 13 ** 3 * 2.0
    if stage == "gather":
        return N_ATOMS * GATHER_POINTS_PER_ATOM * 8.0
    raise ValueError(stage)


# what limits each kernel, from the committed full ncu capture of the
# benchmark workload (profiles/spread_gather_water262k_mixed_full.md)
LIMITER = {
    "gather": "latency and instruction issue at low occupancy (ncu: 500 warp instructions "
              "per atom, 64% issue-active, 16 warps per SM); FP32 lanes are the arithmetic "
              "roofline",
    "spread": "shared-memory integer reductions and instruction issue (ncu: 424 warp "
              "instructions per atom, 74% issue-active, LSU pipe 72% busy)",
}


def fp32_peak(device: int):
    """FP32 fma rate sustained now on this GPU (TFLOP/s), measured by the
    library's own probe kernel (CUDA events, scalar and packed forms)."""
    import ctypes
    from gse_b200 import _lib
    L = _lib.load()
    t, tp = ctypes.c_double(), ctypes.c_double()
    _lib.check(L.gse_measure_fp32_rate(device, None, ctypes.addressof(t), ctypes.addressof(tp)))
    return max(t.value, tp.value), {"scalar_tflops": t.value, "packed_tflops": tp.value}


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
              "timestamp")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.file = None
        self.window = None  # host wall-clock interval of the timed region

    def mark(self, t0: float, t1: float):
        self.window = (t0, t1)

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                if self.window is not None:
                    ts = datetime.datetime.strptime(r[9].strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    if not (self.window[0] <= ts <= self.window[1]):
                        continue
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, name in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def reference_cpu(xyzq64: np.ndarray, box: float, M: int, sigma: float, budget_s: float,
                  max_evals: int):
    """The reference's own CpuGSEk<double,double> (oracle/_ref build) timed on the host."""
    import oracle
    R = oracle.ref()
    n = xyzq64.shape[0]
    h = R.ref_gsek_create(M, M, M, sigma, 0.4, 3.0, 3.0, box, box, box, 332.0716)
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    e = np.zeros(1)
    p = oracle._ptr
    # the reference prints from its spread and gather loops; keep stdout for
    # the JSON line
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    times = []
    try:
        t_start = time.perf_counter()
        while len(times) < max_evals and (not times or time.perf_counter() - t_start < budget_s):
            t0 = time.perf_counter()
            R.ref_gsek_eval(h, n, p(xyzq64), p(e), p(fx), p(fy), p(fz))
            times.append(time.perf_counter() - t0)
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(devnull)
        os.close(saved)
        R.ref_gsek_destroy(h)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": len(times) / sum(times), "evals": len(times), "seconds": sum(times),
            "threads": threads, "energy": float(e[0]), "forces": np.stack([fx, fy, fz], axis=1)}


def parity_vs_reference(F64, E64, Fmx, Emx, Fref, Eref, source):
    """Both GPU forms against the reference's CpuGSEk<double,double> on the same
    box: relative force RMS (Erms, cpu_gse.cpp:131-146) and relative energy."""
    def one(F, E):
        d = F - Fref
        return {"force_rms": float(np.sqrt((d * d).sum() / (Fref * Fref).sum())),
                "energy_rel": abs(E - Eref) / abs(Eref), "source": source}
    return {"fp64": one(F64, E64), "mixed": one(Fmx, Emx)}


def parity_vs_golden(F64, E64, Fmx, Emx):
    """Without the reference build in this run: the committed golden of the
    same box (tests/golden/make_ref_configs.py), 4096 sampled forces."""
    path = os.path.join(ROOT, "tests", "golden", f"ref_{WORKLOAD}.npz")
    if not os.path.exists(path):
        return None
    z = np.load(path)
    idx = z["idx"]
    src = f"the reference's CpuGSEk<double,double> forces of {len(idx)} sampled atoms (golden)"
    return {k: dict(v, source=src) for k, v in
            parity_vs_reference(F64[idx], E64, Fmx[idx], Emx, z["F"], float(z["E"]), src).items()}


def make_workload():
    from gse_b200 import workloads as W
    return W.config_water_262k()


def run_reference_arm(args):
    s = make_workload()
    xyzq = s.xyzq.astype(np.float64)
    import oracle
    kind = "reference" if oracle.have_reference() else "port"
    if kind == "port":
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref was not built (no reference sources)"}))
        return
    budget = float(os.environ.get("GSE_REF_BUDGET_S", "120"))
    # the W warm-up evaluations the other arm takes (plan creation, first touch
    # of the grids), within a budget of their own
    warm = reference_cpu(xyzq, s.box, s.M, s.sigma, 60.0, max(1, args.warmup))
    n_warm = warm["evals"]
    del warm
    r = reference_cpu(xyzq, s.box, s.M, s.sigma, budget, max(1, args.steps))
    sample = (f"{r['evals']} full evaluations of the {s.n}-charge box (of {args.steps} requested "
              f"steps, stopped after a {budget:.0f} s budget); CpuGSEk<double,double> compiled from "
              "the reference sources, spread/gather single-threaded as written, FFTs through the "
              f"project FFTW-API shim on {r['threads']} OpenMP threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": r["evals"], "warmup": n_warm, "ms_per_step": 1000.0 * r["seconds"] / r["evals"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded water-like triplets, 87,381 rigid 3-site molecules)",
        "config": {"workload": WORKLOAD, "n_charges": s.n, "grid": s.M, "box": s.box,
                   "sigma": s.sigma, "kappa": s.kappa, "lambda_sigma1": s.lambda_sigma1,
                   "precision": "fp64 (reference CPU classes)",
                   "parallelism": "host CPU threads of rank 0"},
        "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["threads"], "kind": kind,
                         "sample": sample},
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def gpu_local_cpus(device: int):
    """The CPUs NVML names as local to `device` (read only; nothing is set),
    within this process's allowed set, or None."""
    try:
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(device).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            words = pynvml.nvmlDeviceGetCpuAffinity(h, ((os.cpu_count() or 64) + 63) // 64)
        finally:
            pynvml.nvmlShutdown()
        cpus = {64 * i + b for i, w in enumerate(words) for b in range(64) if (int(w) >> b) & 1}
        cpus &= os.sched_getaffinity(0)
        return cpus or None
    except Exception:
        return None


def bench_batch(steps: int, warmup: int, flush, rank: int = 0, world: int = 1):
    """The batching workload: 256 independent triplet systems, N log-uniform in
    [501, 8001], forward + reverse pass replayed from one CUDA graph after the
    autotuner has picked the launch schedule (per stage or one persistent
    kernel per direction, CTA counts, lanes per atom, work order); the schedule
    it did not keep is timed too, for the record.  With
    several ranks the systems are partitioned across them (no collective on the
    data path); every rank times its share, and the rate is the 256 systems over
    the slowest rank's time.  All ranks must call it."""
    import tempfile

    import torch
    from gse_b200 import multi
    from gse_b200 import workloads as W
    from gse_b200.gse import Batch
    every = W.config_batch(256)
    part = multi.partition_systems([multi.system_cost(y.n, y.grid) for y in every], world)
    syst = [every[i] for i in part[rank]]
    desc = [{"size": y.grid, "box": y.boxes, "n": y.n} for y in syst]
    b = Batch(desc, sigma=2.0, kappa=0.4, lambdaSigma1=3.0)
    xyzq = np.concatenate([y.xyzq for y in syst]).astype(np.float32)
    rng = np.random.default_rng(5)
    G = rng.standard_normal((b.n_total, 3)).astype(np.float32).astype(np.float64)
    b.forward(xyzq)
    cache = os.path.join(tempfile.gettempdir(), f"gse_batch_tune_r{rank}.txt")
    b.autotune(cache, use_cache=False)
    bufs = b.buffers()
    bufs["xyzq"].copy_(torch.from_numpy(xyzq))
    bufs["dLdE"].fill_(1.0)
    bufs["grad_forces"].copy_(torch.from_numpy(np.ascontiguousarray(G.T)))
    stream = torch.cuda.current_stream()
    b.set_stream(stream.cuda_stream)

    def timed_graph():
        """Capture forward + reverse into one graph, replay it `steps` times
        (L2 flushed before each), max over ranks of the mean device time."""
        b.capture(with_adjoint=True)
        for _ in range(warmup):
            b.launch()
        torch.cuda.synchronize()
        multi.barrier()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        for k in range(steps):
            flush.zero_()
            starts[k].record(stream)
            b.launch()
            ends[k].record(stream)
        torch.cuda.synchronize()
        multi.barrier()
        return multi.max_over_ranks(sum(a.elapsed_time(c) for a, c in zip(starts, ends)) / steps,
                                    device=torch.device("cuda", torch.cuda.current_device()))

    def schedule(i):
        if i.fused:
            return {"launches": "one persistent cooperative kernel per direction",
                    "graph_kernel_nodes": int(i.graph_kernels),
                    "gather_lanes_per_atom": int(i.gather_lanes), "ctas": int(i.fused_ctas),
                    "largest_first": bool(i.largest_first)}
        return {"launches": "per stage", "graph_kernel_nodes": int(i.graph_kernels),
                "scatter_ctas": int(i.scatter_ctas), "gather_ctas": int(i.gather_ctas),
                "largest_first": bool(i.largest_first)}

    ms = timed_graph()
    i = b.info()  # after capture: the graph's kernel-node count
    chosen = schedule(i)
    # the schedule the autotuner did not keep, timed the same way for the record
    other = None
    if i.fused_available:
        if i.fused:
            b.set_schedule(fused=False)
        else:
            b.set_schedule(fused=True, gather_lanes=16, largest_first=bool(i.largest_first))
        ms_other = timed_graph()
        other = dict(schedule(b.info()), ms_per_step=ms_other)
    independent = bench_independent(syst, G, min(steps, 5), warmup, flush, stream)
    independent["batch_ms_per_step"] = ms
    n_all = sum(y.n for y in every)
    out = {"workload": "256 independent triplet systems, N log-uniform in [501, 8001], "
                       "M = nearest multiple of 8 to L, sigma 2.0, mixed form",
           "n_total": n_all, "size_classes": int(i.n_size_classes),
           "grid_points": int(i.grid_points), "step": "forward + reverse pass, one CUDA graph",
           "ranks": world, "systems_rank0": len(part[0]),
           "ms_per_step": ms, "systems_per_s": 256 / (ms / 1000.0),
           "charges_per_s": n_all / (ms / 1000.0),
           "autotuned": chosen, "other_schedule": other, "independent": independent}
    b.close()
    return out


def bench_independent(syst, G, steps: int, warmup: int, flush, stream):
    """The batch's work done by separate single-system calls: one mixed
    context per system, its forward (a replayed graph from the second call on)
    and its reverse pass with dL/dE = 1 and the same dL/dF, all systems in
    turn on one stream; device time per step (every system once), L2 flushed
    before each step."""
    import torch
    from gse_b200.gse import Context
    ctxs, args = [], []
    off = 0
    for y in syst:
        c = Context(*y.grid, y.sigma, y.kappa, y.lambda_sigma, y.lambda_sigma1, *y.boxes,
                    precision="mixed")
        c.set_stream(stream.cuda_stream)
        x = torch.from_numpy(np.ascontiguousarray(y.xyzq, dtype=np.float32)).cuda()
        f = torch.empty((3, y.n), dtype=torch.float64, device="cuda")
        e = torch.empty(1, dtype=torch.float64, device="cuda")
        g = torch.from_numpy(np.ascontiguousarray(G[off:off + y.n].T)).cuda()
        d = torch.empty((4, y.n), dtype=torch.float64, device="cuda")
        off += y.n
        ctxs.append(c)
        args.append((y.n, x, f, e, g, d))

    def one_step():
        for c, (n, x, f, e, g, d) in zip(ctxs, args):
            c.forward(n, x, f[0], f[1], f[2], energy_out=e)
            c.adjoint(n, x, 1.0, g[0], g[1], g[2], d[0], d[1], d[2], d[3])

    for _ in range(max(warmup, 2)):  # the second forward call captures the graph
        one_step()
    torch.cuda.synchronize()
    t = 0.0
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        one_step()
        b.record(stream)
        torch.cuda.synchronize()
        t += a.elapsed_time(b)
    launches = sum(c.launch_count() for c in ctxs)
    for c in ctxs:
        c.close()
    return {"step": "every system's gse_forward (graph replay) and gse_adjoint, one context "
                    "per system, one stream", "ms_per_step": t / steps,
            "contexts": len(ctxs), "library_launches_total": int(launches)}


def bench_grid_ops(steps: int, warmup: int, flush, peak: float):
    """The grid operations beside the force path at the benchmark grid (144^3,
    box 140): the on-grid Gaussian convolution of the real-space variant's
    second spreading (sigma2 of sigma 2.0) and the forward-difference field,
    device grids in and out, in both calculation types.  Algorithmic bytes:
    one grid read and one written for the convolution (its two intermediate
    grids, 12 or 24 MB, are the reference's too and largely stay in L2), one
    read and three written for the field."""
    import torch
    from gse_b200.gse import Context
    M, L, sigma = 144, 140.0, 2.0
    s2 = sigma * np.sqrt(1.0 - 2.0 * 0.4)
    rc2 = 3.0 * np.sqrt(2.0) * s2
    out = {"workload": f"grid {M}^3, box {L}, sigma2 {s2:.6f} (sigma {sigma}), device grids"}
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(3)
    for prec, dt in (("mixed", torch.float32), ("fp64", torch.float64)):
        ctx = Context(M, M, M, sigma, 0.4, 3.0, 3.0, L, L, L, precision=prec)
        ctx.set_stream(stream.cuda_stream)
        x = torch.from_numpy(rng.standard_normal((M, M, M))).to(dt).cuda()
        y = torch.empty_like(x)
        E = torch.empty((3, M, M, M), dtype=dt, device="cuda")
        gb = x.numel() * x.element_size() / 1e9

        def timed(fn):
            for _ in range(warmup):
                fn()
            torch.cuda.synchronize()
            t = 0.0
            for _ in range(steps):
                flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn()
                b.record(stream)
                torch.cuda.synchronize()
                t += a.elapsed_time(b)
            return t / steps

        ms_c = timed(lambda: ctx.gauss_spread_on_grid(s2, rc2, L, L, L, x, y))
        ms_e = timed(lambda: ctx.gauss_efield_on_grid(L, L, L, x, E[0], E[1], E[2]))
        out[prec] = {"spread_on_grid_ms": ms_c, "spread_on_grid_gbs": 2 * gb / (ms_c / 1e3),
                     "spread_on_grid_frac_hbm": 2 * gb / (ms_c / 1e3) / peak,
                     "efield_ms": ms_e, "efield_gbs": 4 * gb / (ms_e / 1e3),
                     "efield_frac_hbm": 4 * gb / (ms_e / 1e3) / peak}
        ctx.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference_arm(args)
        return

    import torch
    import torch.distributed as dist
    from gse_b200.gse import Context

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    s = make_workload()
    n = s.n
    stream = torch.cuda.current_stream()

    def make_ctx(precision):
        c = Context(s.M, s.M, s.M, s.sigma, s.kappa, s.lambda_sigma, s.lambda_sigma1, s.box, s.box,
                    s.box, precision=precision, device=local)
        c.set_stream(stream.cuda_stream)
        return c

    def device_inputs(precision):
        ct = np.float32 if precision == "mixed" else np.float64
        x = torch.from_numpy(s.xyzq.astype(ct)).cuda()
        f = torch.empty(3, n, dtype=torch.float64, device="cuda")
        e = torch.empty(1, dtype=torch.float64, device="cuda")
        return x, f, e

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed_loop(ctx, x, f, e, steps, with_timing, clocks=None):
        """Warm-up, then `steps` evaluations each bracketed by CUDA events on the
        launching stream with an L2 flush before each (outside the interval).
        Without stage timing, repeated calls on the same device buffers replay
        the context's captured CUDA graph."""
        for _ in range(args.warmup):
            ctx.forward(n, x, f[0], f[1], f[2], energy_out=e)
        torch.cuda.synchronize()
        ctx.get_timing(reset=True)
        ctx.set_timing(with_timing)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        barrier()
        torch.cuda.synchronize()
        t_busy = None
        if clocks is not None:
            # the sampler needs a moment to start: keep the GPU busy with the
            # same evaluation meanwhile; a timed region of a few ms may fall
            # between two samples, so the clock record spans this busy period
            # and the timed region (same work, back to back)
            clocks.start()
            t_busy = time.time()
            t_end = t_busy + 1.0
            while time.time() < t_end:
                ctx.forward(n, x, f[0], f[1], f[2], energy_out=e)
                torch.cuda.synchronize()
        launches0 = ctx.launch_count()
        t0 = time.time()
        for k in range(steps):
            flush.zero_()  # L2 flush, outside the timed interval
            starts[k].record(stream)
            ctx.forward(n, x, f[0], f[1], f[2], energy_out=e)
            ends[k].record(stream)
        torch.cuda.synchronize()
        t1 = time.time()
        launches = ctx.launch_count() - launches0
        clock_info = None
        if clocks is not None:
            clocks.mark(t_busy, t1)
            clock_info = clocks.stop()
        barrier()
        ctx.set_timing(False)
        stage = ctx.get_timing(reset=True)
        per = [a.elapsed_time(b) for a, b in zip(starts, ends)]
        pct = {"p10": float(np.percentile(per, 10)), "median": float(np.median(per)),
               "p90": float(np.percentile(per, 90))}
        return sum(per), stage, launches, clock_info, pct

    # ---- main arm: requested precision, device-resident inputs ----------
    prec = args.precision
    ctx = make_ctx(prec)
    x, f, e = device_inputs(prec)
    ms_local, _, launches, clock_info, pct = timed_loop(ctx, x, f, e, args.steps, False,
                                                   ClockSampler(local))
    # per-stage device times from a separate, shorter run with stage events
    _, stage, _, _, _ = timed_loop(ctx, x, f, e, max(3, min(args.steps, 20)), True)
    t = torch.tensor([ms_local], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps / (ms_max / 1000.0)
    F_main = f.clone()
    E_main = float(e.item())

    # ---- e2e: public call with pinned host buffers ----------------------
    # the page-locked buffers are placed on the host memory next to the GPU:
    # allocated while this thread runs on the GPU's local CPUs (NVML's
    # affinity, read only), then the thread's affinity is put back
    ct = np.float32 if prec == "mixed" else np.float64
    near_cpus = gpu_local_cpus(torch.cuda.current_device())
    before = os.sched_getaffinity(0)
    if near_cpus:
        os.sched_setaffinity(0, near_cpus)
    # filled by one numpy assignment: a buffer filled by torch's pin_memory()
    # copy was read by the GPU at 15 GB/s instead of 51 until the host caches
    # had turned over (`pcie` below times both)
    hx = torch.empty(s.xyzq.shape, dtype=torch.float32 if ct is np.float32 else torch.float64,
                     pin_memory=True)
    hx.numpy()[:] = s.xyzq.astype(ct)
    hf = torch.empty(3, n, dtype=torch.float64, pin_memory=True)
    if near_cpus:
        os.sched_setaffinity(0, before)
    hxn, hfn = hx.numpy(), hf.numpy()
    for _ in range(args.warmup):
        ctx.forward(n, hxn, hfn[0], hfn[1], hfn[2])
    e2e_steps = max(3, min(args.steps, 20))
    barrier()
    torch.cuda.synchronize()
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(e2e_steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(e2e_steps)]
    for k in range(e2e_steps):
        flush.zero_()
        ev0[k].record(stream)
        ctx.forward(n, hxn, hfn[0], hfn[1], hfn[2])
        ev1[k].record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = sum(a.elapsed_time(b) for a, b in zip(ev0, ev1))
    t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * e2e_steps / (float(t.item()) / 1000.0)
    h2d = n * 4 * np.dtype(ct).itemsize
    d2h = 3 * n * 8 + 8
    # the same two copies alone, on this box's link, to explain e2e (which
    # varies from box to box with the host link while the device time does not)
    dx = torch.empty(hx.shape, dtype=hx.dtype, device="cuda")
    df = torch.empty(hf.shape, dtype=hf.dtype, device="cuda")

    def copy_ms(fn):
        a = [torch.cuda.Event(enable_timing=True) for _ in range(e2e_steps)]
        b = [torch.cuda.Event(enable_timing=True) for _ in range(e2e_steps)]
        for k in range(e2e_steps):
            a[k].record(stream)
            fn()
            b[k].record(stream)
        torch.cuda.synchronize()
        return sorted(x.elapsed_time(y) for x, y in zip(a, b))[e2e_steps // 2]

    ms_h2d = copy_ms(lambda: dx.copy_(hx, non_blocking=True))
    ms_d2h = copy_ms(lambda: hf.copy_(df, non_blocking=True))
    # the upload from a buffer filled by torch's pin_memory() copy instead
    hx2 = torch.from_numpy(s.xyzq.astype(ct)).pin_memory()
    ms_h2d2 = copy_ms(lambda: dx.copy_(hx2, non_blocking=True))
    bx, bf = hx.numel() * hx.element_size(), hf.numel() * hf.element_size()
    pcie = {"what": "the evaluation's position upload and force download alone, pinned host "
                    "memory, median of the e2e step count",
            "host_buffers": (f"allocated on the {len(near_cpus)} CPUs local to the GPU"
                             if near_cpus else "default placement (no GPU-local CPU set found)"),
            "h2d_ms": ms_h2d, "d2h_ms": ms_d2h,
            "h2d_gbs": bx / (ms_h2d * 1e6), "d2h_gbs": bf / (ms_d2h * 1e6),
            "h2d_gbs_pin_memory_copy": bx / (ms_h2d2 * 1e6),
            "device_ms_plus_copies": ms_max / args.steps + ms_h2d + ms_d2h,
            "e2e_ms": float(t.item()) / e2e_steps}

    # ---- the other precision, for the mixed-vs-FP64 comparison ----------
    other = "fp64" if prec == "mixed" else "mixed"
    ctx2 = make_ctx(other)
    x2, f2, e2 = device_inputs(other)
    ms2, _, _, _, _ = timed_loop(ctx2, x2, f2, e2, max(3, min(args.steps, 50)), False)
    value2 = world * max(3, min(args.steps, 50)) / (ms2 / 1000.0)
    F64 = (f2 if other == "fp64" else F_main).double().cpu().numpy().T
    Fmx = (F_main if other == "fp64" else f2).double().cpu().numpy().T
    E64 = float(e2.item()) if other == "fp64" else E_main
    Emx = E_main if other == "fp64" else float(e2.item())
    d = Fmx - F64
    force_rms = float(np.sqrt((d * d).sum() / (F64 * F64).sum()))
    energy_rel = abs(Emx - E64) / abs(E64)

    # accuracy of both forms against the FP64 Ewald reciprocal sum (converged k cut)
    accuracy = None
    if rank == 0:
        from gse_b200.gse import ewald_kcut, ewald_recip
        kc = ewald_kcut(s.sigma, s.boxes)
        t0 = time.perf_counter()
        e_ew, f_ew = ewald_recip(s.sigma, kc, s.boxes, s.xyzq.astype(np.float64), device=local)
        t_ew = time.perf_counter() - t0

        def rel_rms(F):
            dd = F - f_ew
            return float(np.sqrt((dd * dd).sum() / (f_ew * f_ew).sum()))

        accuracy = {"oracle": f"FP64 Ewald reciprocal sum on the GPU, kcut {kc}",
                    "oracle_seconds": t_ew,
                    "mixed": {"force_rms": rel_rms(Fmx), "energy_rel": abs(Emx - e_ew) / abs(e_ew)},
                    "fp64": {"force_rms": rel_rms(F64), "energy_rel": abs(E64 - e_ew) / abs(e_ew)}}
        # the whole Ewald sum: the same direct (real-space) sum beside GSE-k and
        # beside the Ewald reciprocal sum (rcut 9, as the reference's drivers use;
        # no exclusions, as GSE-k's k-space sum has none); the direct sum returns
        # the gradient dE/dx, GSE-k and the reciprocal sum the force -dE/dx
        from gse_b200.gse import ewald_direct
        t0 = time.perf_counter()
        e_dir, g_dir = ewald_direct(s.sigma, 9.0, s.boxes, s.xyzq.astype(np.float64), device=local)
        t_dir = time.perf_counter() - t0
        f_tot = f_ew - g_dir

        def tot_err(F, E):
            dd = F - f_ew
            return {"force_rms": float(np.sqrt((dd * dd).sum() / (f_tot * f_tot).sum())),
                    "energy_rel": abs(E - e_ew) / abs(e_dir + e_ew)}

        accuracy["total"] = {"oracle": f"FP64 Ewald direct (rcut 9.0) + reciprocal (kcut {kc}) "
                                       "sums on the GPU; GSE-k with the same direct sum",
                             "direct_seconds": t_dir,
                             "mixed": tot_err(Fmx, Emx), "fp64": tot_err(F64, E64)}

    # the batched workload, partitioned across the ranks (every rank takes part)
    batch = None
    if not args.no_batch:
        try:
            batch = bench_batch(max(3, min(args.steps, 20)), args.warmup, flush, rank, world)
        except Exception as exc:  # noqa: BLE001
            if world > 1:
                raise  # the other ranks wait in its collectives: fail the job
            batch = {"failed": str(exc)}

    if rank == 0:
        # roofline of the dominant kernel
        peak, peak_kind = hbm_peak()
        dom = max(("spread", "gather"), key=lambda k: stage[k][0] / max(stage[k][1], 1))
        dom_ms = stage[dom][0] / max(stage[dom][1], 1)
        ab = algorithmic_bytes(dom, prec)
        achieved = ab / (dom_ms / 1000.0) / 1e9
        af = algorithmic_flops(dom)
        achieved_tf = af / (dom_ms / 1000.0) / 1e12
        try:
            fpeak, fpeak_forms = fp32_peak(local)
        except Exception as exc:  # noqa: BLE001
            fpeak, fpeak_forms = None, {"failed": str(exc)}
        traffic = None
        prof = os.path.join(ROOT, "profiles", "traffic_water262k.txt")
        if os.path.exists(prof):
            with open(prof) as fh:
                for ln in fh:
                    parts = ln.split()
                    if len(parts) == 3 and parts[0] == dom and parts[1] == prec:
                        traffic = int(parts[2])
        cpu = None
        ref_parity = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                import oracle
                if oracle.have_reference():
                    r = reference_cpu(s.xyzq.astype(np.float64), s.box, s.M, s.sigma, 12.0, 3)
                    ref_parity = parity_vs_reference(F64, E64, Fmx, Emx, r["forces"], r["energy"],
                                                     "CpuGSEk<double,double> forces of every "
                                                     "atom, computed in this run")
                    cpu = {"value": r["value"], "unit": UNIT, "cores": r["threads"],
                           "kind": "reference",
                           "sample": f"{r['evals']} full evaluations of the same {n}-charge box "
                                     "by CpuGSEk<double,double> compiled from the reference "
                                     "sources (spread/gather single-threaded as written; FFTs "
                                     f"through the FFTW-API shim on {r['threads']} threads)"}
            except Exception as exc:  # noqa: BLE001
                cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                       "sample": f"failed: {exc}"}
        if ref_parity is None:
            ref_parity = parity_vs_golden(F64, E64, Fmx, Emx)
        grid_ops = None
        if not args.no_batch:
            try:
                grid_ops = bench_grid_ops(max(3, min(args.steps, 20)), args.warmup, flush, peak)
            except Exception as exc:  # noqa: BLE001
                grid_ops = {"failed": str(exc)}
        per_stage = {k: round(v[0] / max(v[1], 1), 4) for k, v in stage.items()}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec == "mixed" else "f64",
            "data": "synthetic (seeded water-like triplets, 87,381 rigid 3-site molecules)",
            "config": {"workload": WORKLOAD, "n_charges": n, "grid": s.M, "box": s.box,
                       "sigma": s.sigma, "kappa": s.kappa, "lambda_sigma1": s.lambda_sigma1,
                       "precision": prec, "parallelism": f"replicas{world}",
                       "l2": "flushed between timed evaluations (256 MiB write)"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "pcie": pcie,
            "gpu_launches": int(launches),
            "roofline": {"bound": "fp32", "achieved": achieved_tf, "peak": fpeak,
                         "unit": "TFLOP/s", "frac": achieved_tf / fpeak if fpeak else None,
                         "traffic": traffic, "kernel": dom,
                         "peak_source": "measured in this run (gse_measure_fp32_rate)",
                         "peak_forms": fpeak_forms, "algorithmic_flops_per_launch": af,
                         "launch_ms": dom_ms, "limiter": LIMITER.get(dom),
                         "hbm": {"achieved": achieved, "peak": peak, "unit": "GB/s",
                                 "frac": achieved / peak, "peak_source": peak_kind,
                                 "algorithmic_bytes_per_launch": ab}},
            "cpu_baseline": cpu,
            "clocks": clock_info,
            "stage_ms": per_stage,
            "eval_ms_percentiles": {k: round(v, 4) for k, v in pct.items()},
            f"{other}_value": value2,
            "mixed_vs_fp64": {"force_rms": force_rms, "energy_rel": energy_rel},
            "fp64_vs_reference": ref_parity and ref_parity["fp64"],
            "mixed_vs_reference": ref_parity and ref_parity["mixed"],
            "vs_ewald": accuracy,
            "energy": E_main,
            "batch": batch,
            "grid_ops": grid_ops,
        }
        print(json.dumps(line), flush=True)

    del ctx, ctx2
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
