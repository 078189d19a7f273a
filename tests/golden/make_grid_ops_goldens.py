"""Generate golden vectors for the grid operations of CpuGaussCharge beside
the force path, from the reference's own CPU class:

  rhoS        spreadChargeOnGrid(sigma, rcut, box, rho, rhoS)  (CpuGaussCharge.cpp:390-519)
  Ex, Ey, Ez  calcElectricFieldOnGrid(box, phi, Ex, Ey, Ez)    (CpuGaussCharge.cpp:62-98)
  dip         calcDipoleSum(box, rho, dx, dy, dz)              (CpuGaussCharge.cpp:188-226)

for <double,double> ("d") and <double,float> ("f").  Runs in the container
that holds the reference sources (it builds oracle/_ref/libgse_ref.so).

Cases: seeded normal grids with odd, even and non-cubic sizes; a stencil
wider than the grid (2n+1 = 13 > 9); and the GSE-r second spreading step,
rho = spreadChargeToGrid(sigma1) of 150 water-like triplets convolved with
sigma2 (CpuGSEr.cpp:39-42).  The potential fed to the field is the input grid.

Output: tests/golden/grid_ops_goldens.npz.
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
    rng = np.random.default_rng(7)
    out = []
    for name, M, box, sigma in (("rand_12x10x14", (12, 10, 14), (11.0, 9.5, 13.0), 0.9),
                                ("rand_11cube", (11, 11, 11), (11.7, 11.7, 11.7), 0.894427191),
                                ("rand_9cube_wide", (9, 9, 9), (9.0, 9.0, 9.0), 1.2)):
        out.append((name, M, box, sigma, rng.standard_normal(M[::-1])))
    M, box = (12, 14, 16), (12.0, 13.2, 14.4)
    s1, s2, rc1 = oracle.gse_params(2.0)
    x = W.triplets(150, 12.0, 2).astype(np.float64) * np.array([1.0, 1.1, 1.2, 1.0])
    rho = oracle.ref_spread(M, box, s1, rc1, x, dtype=np.float64)
    out.append(("gser_water150", M, box, s2, rho))
    return out


def main():
    oracle.build(with_reference=True)
    data = {}
    for name, M, box, sigma, rho in cases():
        rcut = 3.0 * np.sqrt(2.0) * sigma
        p = name + "/"
        data[p + "M"] = np.array(M)
        data[p + "box"] = np.array(box)
        data[p + "sigma"] = np.array(sigma)
        data[p + "rcut"] = np.array(rcut)
        for sfx, dt in (("d", np.float64), ("f", np.float32)):
            r = rho.astype(dt)
            data[p + "rho_" + sfx] = r
            data[p + "rhoS_" + sfx] = oracle.ref_spread_on_grid(M, box, sigma, rcut, r, dt)
            ex, ey, ez = oracle.ref_efield(M, box, r, dt)
            data[p + "Ex_" + sfx], data[p + "Ey_" + sfx], data[p + "Ez_" + sfx] = ex, ey, ez
            data[p + "dip_" + sfx] = oracle.ref_dipole_sum(M, box, r, dt)
        print(name, M, data[p + "dip_d"])
    np.savez_compressed(os.path.join(HERE, "grid_ops_goldens.npz"), **data)


if __name__ == "__main__":
    main()
