"""Generate golden vectors from the reference's own CPU classes.

Runs in the container that holds the reference sources: it builds
oracle/_ref/libgse_ref.so (the reference's CpuGSEk / CpuGaussCharge /
CpuGreensFuncGSE compiled unchanged, FFTs through the FFTW-API shim) and
records, per case, the inputs and the reference outputs:

  E, F          CpuGSEk<double,double>: spreadCharge1 -> solvePoisson ->
                calculateEnergy -> interpolateForce (cpu_gse.cpp:440-455)
  rhoS, phi     the reference's grids (small grids only)
  rho_f         CpuGaussCharge<double,float>::spreadChargeToGrid
  F_f           CpuGaussCharge<double,float>::interpolateForce from phi (float)
  rho_norm      spreadChargeToGrid(normalize=true) in double

Output: tests/golden/gse_goldens.npz (+ water_23559.npz for the 23,559-charge
water box, energy and forces only).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from gse_b200 import workloads as W  # noqa: E402


def cases():
    out = []
    out.append(("pair_L20_M20", W.pair(1.0, 20.0, 1), (20, 20, 20), (20.0, 20.0, 20.0), 2.121320344))
    out.append(("refpair_L20_M20", W.reference_pair(1.0), (20, 20, 20), (20.0, 20.0, 20.0),
                2.121320344))
    out.append(("random64_L16_M16", W.random_charges(64, 16.0, 1), (16, 16, 16),
                (16.0, 16.0, 16.0), 2.0))
    out.append(("water300_noncubic", W.triplets(300, 15.0, 2).astype(np.float64) *
                np.array([1.0, 1.1, 1.2, 1.0]), (16, 18, 20), (15.0, 16.5, 18.0), 2.0))
    out.append(("water600_L18_M17_odd", W.triplets(600, 18.0, 3).astype(np.float64), (17, 17, 17),
                (18.0, 18.0, 18.0), 2.0))
    # the stencil is wider than the grid (2n+1 = 13 > M = 10): multiple wrap-around
    out.append(("water96_L9_M10_wide", W.triplets(96, 9.0, 4).astype(np.float64), (10, 10, 10),
                (9.0, 9.0, 9.0), 2.0))
    return out


def main():
    oracle.build(with_reference=True)
    data = {}
    for name, xyzq, M, box, sigma in cases():
        xyzq = np.ascontiguousarray(xyzq, dtype=np.float64)
        s1, s2, rc = oracle.gse_params(sigma)
        E, F, rho, phi = oracle.ref_gsek_forward(M, box, sigma, xyzq, want_grids=True)
        xf = xyzq.astype(np.float32)
        rho_f = oracle.ref_spread(M, box, s1, rc, xf, dtype=np.float32)
        Ff = np.stack(oracle.ref_gather(M, box, s1, rc, xf, phi.astype(np.float32),
                                        dtype=np.float32), axis=1)
        rho_n = oracle.ref_spread(M, box, s1, rc, xyzq, dtype=np.float64, normalize=True)
        p = name + "/"
        data[p + "xyzq"] = xyzq
        data[p + "M"] = np.array(M)
        data[p + "box"] = np.array(box)
        data[p + "sigma"] = np.array(sigma)
        data[p + "E"] = np.array(E)
        data[p + "F"] = F
        data[p + "rhoS"] = rho
        data[p + "phi"] = phi
        data[p + "rho_f"] = rho_f
        data[p + "F_f"] = Ff
        data[p + "rho_norm"] = rho_n
        print(name, E)
    np.savez_compressed(os.path.join(HERE, "gse_goldens.npz"), **data)

    s = W.config_water_23k()
    xyzq = s.xyzq.astype(np.float64)
    E, F = oracle.ref_gsek_forward(s.grid, s.boxes, s.sigma, xyzq)
    np.savez_compressed(os.path.join(HERE, "water_23559.npz"), E=np.array(E), F=F,
                        M=np.array(s.grid), box=np.array(s.boxes), sigma=np.array(s.sigma),
                        xyzq_sha=np.frombuffer(__import__("hashlib").sha256(
                            s.xyzq.tobytes()).digest(), dtype=np.uint8))
    print("water_23559", E)


if __name__ == "__main__":
    main()
