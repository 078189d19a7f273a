"""Seeded synthetic charge systems for the GSE-k path.

The reference drives GSE-k with a two-charge pair (cpu_gse.cpp:638-700), with
uniformly random +-1 charges (cpu_gse.cpp:423-438) and with a 48k-atom water
box read from disk (cpu_gse.cpp:216-229).  The workloads here are seeded
stand-ins with those shapes: rigid 3-site neutral water-like triplets
(O -0.834 at the centre, two H +0.417 at 0.9572 A with a 104.52 degree H-O-H
angle), centres uniform in the box and orientations uniform random rotations.
Positions are generated in FP32 (the mixed path's input type); the FP64 path
uses the same values widened.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List

import numpy as np

Q_O = -0.834
Q_H = 0.417
R_OH = 0.9572
ANGLE_HOH_DEG = 104.52


@dataclass
class System:
    """One periodic cubic system: positions+charges and grid parameters."""

    name: str
    xyzq: np.ndarray  # (n, 4) float32 AoS {x, y, z, q}
    box: float
    M: int
    sigma: float
    kappa: float = 0.4
    lambda_sigma: float = 3.0
    lambda_sigma1: float = 3.0

    @property
    def n(self) -> int:
        return int(self.xyzq.shape[0])

    @property
    def boxes(self):
        return (self.box, self.box, self.box)

    @property
    def grid(self):
        return (self.M, self.M, self.M)


def _random_rotations(rng: np.random.Generator, k: int) -> np.ndarray:
    """k uniform random rotation matrices (normalised Gaussian quaternions)."""
    q = rng.standard_normal((k, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.empty((k, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def triplets(n_atoms: int, box: float, seed: int = 1) -> np.ndarray:
    """n_atoms (a multiple of 3) water-like triplet charges in a cubic box."""
    if n_atoms % 3 != 0:
        raise ValueError("triplet systems need a multiple of 3 charges")
    k = n_atoms // 3
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, box, size=(k, 3))
    R = _random_rotations(rng, k)
    half = math.radians(ANGLE_HOH_DEG) / 2.0
    body = np.array([[0.0, 0.0, 0.0],
                     [R_OH * math.sin(half), R_OH * math.cos(half), 0.0],
                     [-R_OH * math.sin(half), R_OH * math.cos(half), 0.0]])
    pos = centres[:, None, :] + np.einsum("kij,sj->ksi", R, body)
    out = np.empty((k, 3, 4), dtype=np.float32)
    out[:, :, :3] = pos
    out[:, 0, 3] = Q_O
    out[:, 1:, 3] = Q_H
    return out.reshape(-1, 4)


def pair(r: float = 1.0, box: float = 20.0, seed: int = 1) -> np.ndarray:
    """Charges -1 (box centre) and +1 at distance r along a seeded direction."""
    rng = np.random.default_rng(seed)
    u = rng.standard_normal(3)
    u /= np.linalg.norm(u)
    c = np.full(3, 0.5 * box)
    out = np.zeros((2, 4), dtype=np.float64)
    out[0, :3] = c
    out[0, 3] = -1.0
    out[1, :3] = c + r * u
    out[1, 3] = 1.0
    return out


def reference_pair(r: float = 1.0) -> np.ndarray:
    """testPair's geometry (cpu_gse.cpp:689-698): -1 at the origin, +1 at (a,a,a), a=r/sqrt(3)."""
    a = r / math.sqrt(3.0)
    return np.array([[0.0, 0.0, 0.0, -1.0], [a, a, a, 1.0]], dtype=np.float64)


def random_charges(n: int, box: float, seed: int = 1) -> np.ndarray:
    """testRandom's layout (cpu_gse.cpp:430-436): uniform positions, alternating -1/+1."""
    rng = np.random.default_rng(seed)
    out = np.empty((n, 4), dtype=np.float64)
    out[:, :3] = rng.uniform(0.0, box, size=(n, 3))
    out[:, 3] = (np.arange(n) % 2) * 2 - 1
    return out


def triplet_exclusions(n_atoms: int):
    """Exclusion lists of rigid 3-site molecules in CHARMM's format, as
    CpuEwaldDirect::setupExclusions reads them (CpuEwaldDirect.cpp:31-40):
    iblo14[a] is the cumulative end of atom a's entries in inb14, whose
    entries are 1-based partners.  Each molecule (O, H, H) lists O-H1 and
    O-H2 under O and H1-H2 under H1; an atom left over after the last whole
    molecule has none."""
    iblo14 = np.zeros(n_atoms, dtype=np.int32)
    inb14 = []
    for a in range(n_atoms):
        m0 = a - a % 3
        if m0 + 2 < n_atoms:
            inb14.extend(b + 1 for b in range(a + 1, m0 + 3))
        iblo14[a] = len(inb14)
    return iblo14, np.array(inb14, dtype=np.int32)


# --------------------------------------------------------------------------
# Named workloads (sizes as the GSE-k benchmark configurations state them)
# --------------------------------------------------------------------------
def config_pair() -> System:
    return System("pair_L20_M20", pair(1.0, 20.0, 1), 20.0, 20, 2.121320344)


def config_water_23k() -> System:
    return System("water_23559_L62.23_M64", triplets(23559, 62.23, 1), 62.23, 64, 2.0)


def config_water_262k() -> System:
    """262,144 charges requested; 262,143 = 87,381 triplets (262,144 is not a multiple of 3)."""
    return System("water_262143_L140_M144", triplets(262143, 140.0, 1), 140.0, 144, 2.0)


def config_water_48k() -> System:
    return System("water_48000_L78.4_M80", triplets(48000, 78.4, 1), 78.4, 80, 2.0)


def config_batch(num_systems: int = 256, seed: int = 1, density: float = 0.0978,
                 n_min: int = 501, n_max: int = 8001) -> List[System]:
    """Uneven batch: N_s log-uniform in [n_min, n_max] (multiple of 3),
    L_s = (N_s/density)^(1/3), M_s = nearest multiple of 8 to L_s."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(num_systems):
        n = 3 * int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max))) / 3.0))
        L = (n / density) ** (1.0 / 3.0)
        M = max(8, 8 * int(round(L / 8.0)))
        out.append(System(f"batch{s}_n{n}", triplets(n, L, seed * 100003 + s), L, M, 2.0))
    return out
