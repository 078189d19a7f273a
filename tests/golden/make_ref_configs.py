"""Golden outputs of the reference's CpuGSEk<double,double> on the two large
synthetic water boxes of the benchmark configurations:

  water_262143_L140_M144  87,381 rigid triplets, box 140, grid 144, sigma 2.0
                          (the box the force-evaluation rate is quoted on)
  water_48000_L78.4_M80   16,000 rigid triplets, box 78.4, grid 80, sigma 2.0
                          (the differentiation configuration's forward)

kappa 0.4, lambdaSigma = lambdaSigma1 = 3.0.  The inputs are regenerated from
their seed by gse_b200.workloads (FP32 positions, widened to double for the
reference); the sha256 of the widened array is stored so a test can confirm it
regenerated the same input.  The reference classes are the ones compiled from
its sources (oracle/_ref/libgse_ref.so; FFTs through the FFTW-API shim):
spreadCharge1 -> solvePoisson -> calculateEnergy -> interpolateForce
(CpuGSEk.cpp:30-58, CpuGSE.cpp:70-103).

Runs in the container that holds the reference sources.  Writes, per box,
ref_<name>.npz with E; the forces of 4096 atoms (a seeded sample, indices in
`idx`); sum F and sum |F|^2 over all atoms; the input's sha256.
"""
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from gse_b200 import workloads as W  # noqa: E402

SAMPLE = 4096


def input_sha(x64: np.ndarray) -> np.ndarray:
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(x64).tobytes()).digest(), np.uint8)


def make(system, seed: int) -> None:
    x = system.xyzq.astype(np.float64)
    t0 = time.perf_counter()
    E, F = oracle.ref_gsek_forward(system.grid, system.boxes, system.sigma, x,
                                   kappa=system.kappa, lambda_sigma=system.lambda_sigma,
                                   lambda_sigma1=system.lambda_sigma1)
    dt = time.perf_counter() - t0
    idx = np.sort(np.random.default_rng(seed).choice(x.shape[0], SAMPLE, replace=False))
    out = os.path.join(HERE, f"ref_{system.name}.npz")
    np.savez_compressed(out, E=np.array(E), idx=idx, F=F[idx], Fsum=F.sum(axis=0),
                        F2sum=np.array((F * F).sum()), xyzq_sha=input_sha(x),
                        sigma=np.array(system.sigma), box=np.array(system.box),
                        grid=np.array(system.M), n=np.array(x.shape[0]))
    print(f"{system.name}: E={E!r} F2sum={(F * F).sum()!r} ({dt:.1f} s) -> {out}")


def main():
    if oracle.reference_dir() is None:
        sys.exit("the reference sources are needed (set GSE_REFERENCE_DIR)")
    oracle.build(with_reference=True)
    make(W.config_water_262k(), 262)
    make(W.config_water_48k(), 48)


if __name__ == "__main__":
    main()
