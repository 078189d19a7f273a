"""Small, self-ending GPU cases to run under a profiler (ncu), one GPU.

  python profile_cases.py forward [--evals 3] [--precision mixed|fp64]
      the benchmark workload (262,143 water-like charges, M = 144, sigma 2):
      one context, `evals` forward evaluations on device buffers (the first
      builds the Green's table and records the key, the next ones run
      directly and then replay a CUDA graph), no L2-flush buffer
  python profile_cases.py gridops [--steps 5] [--warmup 2]
      the bench's grid-operation leg (on-grid convolution and field of a 144^3
      grid, both calculation types)

Each prints one line (the energy, or the grid-operation timings as JSON) and
exits; the device memory held stays at a few hundred MB.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def forward(evals: int, precision: str) -> None:
    import numpy as np
    import torch

    from gse_b200 import workloads as W
    from gse_b200.gse import Context
    s = W.config_water_262k()
    n = s.n
    ctx = Context(s.M, s.M, s.M, s.sigma, s.kappa, s.lambda_sigma, s.lambda_sigma1, s.box, s.box,
                  s.box, precision=precision)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    ct = np.float32 if precision == "mixed" else np.float64
    x = torch.from_numpy(s.xyzq.astype(ct)).cuda()
    f = torch.empty(3, n, dtype=torch.float64, device="cuda")
    e = torch.empty(1, dtype=torch.float64, device="cuda")
    for _ in range(evals):
        ctx.forward(n, x, f[0], f[1], f[2], energy_out=e)
    torch.cuda.synchronize()
    print("E", e.item())


def gridops(steps: int, warmup: int) -> None:
    import torch
    import bench
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    peak, _ = bench.hbm_peak()
    print(json.dumps(bench.bench_grid_ops(steps, warmup, flush, peak)))


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(prog="python profile_cases.py")
    sub = ap.add_subparsers(dest="case", required=True)
    fw = sub.add_parser("forward")
    fw.add_argument("--evals", type=int, default=3)
    fw.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    go = sub.add_parser("gridops")
    go.add_argument("--steps", type=int, default=5)
    go.add_argument("--warmup", type=int, default=2)
    a = ap.parse_args(argv)
    if a.case == "forward":
        forward(a.evals, a.precision)
    else:
        gridops(a.steps, a.warmup)


if __name__ == "__main__":
    main()
