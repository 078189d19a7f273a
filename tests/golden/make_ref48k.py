"""Golden outputs of the reference's own real-system GSE-k case, test48K
(cpu_gse.cpp:216-250): the 48,191 charges of data/xyzq_48k.txt, sigma
2.12132034355964, kappa 0.4, lambdaSigma = lambdaSigma1 = 3.0, box 80, grid 80,
CpuGSEk<double,double> (spreadCharge1 -> solvePoisson -> calculateEnergy ->
interpolateForce), computed by the reference's classes compiled from its
sources (oracle/_ref/libgse_ref.so; FFTs through the FFTW-API shim).

Runs in the container that holds the reference sources.  Writes

  xyzq_48k.txt.xz  the input file itself, xz-compressed; float() of each token
                   gives the double the reference's istream >> gives (both round
                   the decimal text correctly)
  ref48k.npz       E; the forces of 3000 atoms (a seeded sample, indices in
                   `idx`); sum F and sum |F|^2 over all atoms; the sha256 of the
                   parsed input array
"""
import hashlib
import lzma
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

REF_DATA = os.path.join(os.environ.get("GSE_REFERENCE_DIR", "/root/reference"), "data",
                        "xyzq_48k.txt")
SIGMA, BOX, GRID = 2.12132034355964, 80.0, 80


def load_xz(path):
    """The 48k input from its xz copy, as float64 [n, 4]."""
    with lzma.open(path, "rt") as f:
        return np.array([float(t) for t in f.read().split()], dtype=np.float64).reshape(-1, 4)


def main():
    oracle.build(with_reference=True)
    text = open(REF_DATA, "rb").read()
    xz = os.path.join(HERE, "xyzq_48k.txt.xz")
    with lzma.open(xz, "wb", preset=9) as f:
        f.write(text)
    x = load_xz(xz)
    assert x.shape == (48191, 4)
    E, F = oracle.ref_gsek_forward((GRID,) * 3, (BOX,) * 3, SIGMA, x)
    idx = np.sort(np.random.default_rng(48).choice(x.shape[0], 3000, replace=False))
    np.savez_compressed(os.path.join(HERE, "ref48k.npz"), E=np.array(E), idx=idx, F=F[idx],
                        Fsum=F.sum(axis=0), F2sum=np.array((F * F).sum()),
                        xyzq_sha=np.frombuffer(hashlib.sha256(x.tobytes()).digest(), np.uint8),
                        sigma=np.array(SIGMA), box=np.array(BOX), grid=np.array(GRID))
    print("E", E, "F2sum", (F * F).sum())


if __name__ == "__main__":
    main()
