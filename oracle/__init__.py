"""CPU oracle for the GSE-k reciprocal-space path (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package.  It wraps two shared libraries built by
``oracle/Makefile``:

* ``libgse_oracle.so`` -- the project's C restatement of the reference path
  (``gse_oracle.c``; each function cites the ap-hynninen/GSE file:line it
  restates);
* ``_ref/libgse_ref.so`` -- the reference's own CpuGSEk / CpuGaussCharge /
  CpuGreensFuncGSE / CpuEwaldRecip / CpuEwaldDirect classes compiled unchanged
  from the reference sources, linked with an FFTW-API shim.  It is optional:
  it exists where the reference sources were available at build time.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libgse_oracle.so")
_REF_PATH = os.path.join(_HERE, "_ref", "libgse_ref.so")

CCELEC = 332.0716

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double

_lib = None
_ref = None


# Where the reference sources are read from when oracle/_ref is built: the
# GSE_REFERENCE_DIR environment variable, else the build container's checkout.
DEFAULT_REFERENCE_DIR = "/root/reference"


def reference_dir() -> Optional[str]:
    """The reference source tree, or None where it is absent (a GPU box uses
    the prebuilt oracle/_ref)."""
    d = os.environ.get("GSE_REFERENCE_DIR", DEFAULT_REFERENCE_DIR)
    return d if os.path.isfile(os.path.join(d, "CpuGSEk.cpp")) else None


def build(with_reference: bool = False) -> None:
    """Compile the restatement (and, if asked, the reference build from
    reference_dir())."""
    cmd = ["make", "-s", "-C", _HERE]
    if with_reference and reference_dir():
        cmd += ["ref", f"REF={reference_dir()}"]
    else:
        cmd += ["all"]
    subprocess.run(cmd, check=True)


def _ptr(a: Optional[np.ndarray], kind=_dp):
    if a is None:
        return ctypes.cast(None, kind)
    return a.ctypes.data_as(kind)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build(False)
        L = ctypes.CDLL(_LIB_PATH)
        for sfx, p in (("d", _dp), ("f", _fp)):
            f = getattr(L, f"orc_spread_{sfx}")
            f.argtypes = [_i, _i, _i, _d, _d, _i, p, _d, _d, _d, _i, p]
            f.restype = _i
            f = getattr(L, f"orc_gather_{sfx}")
            f.argtypes = [_i, _i, _i, _d, _d, _i, p, _d, _d, _d, p, _dp, _dp, _dp]
            f.restype = _i
            f = getattr(L, f"orc_green_mul_{sfx}")
            f.argtypes = [_i, _i, _i, _d, _d, _d, _d, p]
            f.restype = None
            f = getattr(L, f"orc_energy_{sfx}")
            f.argtypes = [_i, _i, _i, _d, _d, _d, _d, p, p]
            f.restype = _d
            f = getattr(L, f"orc_spread_on_grid_{sfx}")
            f.argtypes = [_i, _i, _i, _d, _d, _d, _d, _d, p, p]
            f.restype = _i
            f = getattr(L, f"orc_efield_{sfx}")
            f.argtypes = [_i, _i, _i, _d, _d, _d, p, p, p, p]
            f.restype = None
            f = getattr(L, f"orc_dipole_{sfx}")
            f.argtypes = [_i, _i, _i, _d, _d, _d, p, _dp]
            f.restype = None
        L.orc_fft_r2c_3d.argtypes = [_i, _i, _i, _dp, _dp]
        L.orc_fft_r2c_3d.restype = _i
        L.orc_fft_c2r_3d.argtypes = [_i, _i, _i, _dp, _dp]
        L.orc_fft_c2r_3d.restype = _i
        L.orc_gsek_forward_d.argtypes = [_i, _i, _i, _d, _d, _d, _d, _d, _d, _d, _i, _dp,
                                         _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_gsek_forward_d.restype = _i
        L.orc_ewald_recip.argtypes = [_d, _i, _d, _d, _d, _d, _i, _dp, _dp, _dp, _dp]
        L.orc_ewald_recip.restype = _d
        L.orc_ewald_direct.argtypes = [_d, _d, _d, _d, _d, _d, _i, _dp, _i, _ip, _ip, _dp, _dp,
                                       _dp]
        L.orc_ewald_direct.restype = _d
        _lib = L
    return _lib


def have_reference() -> bool:
    return os.path.exists(_REF_PATH)


def ref():
    """The reference's own classes (oracle/_ref/libgse_ref.so)."""
    global _ref
    if _ref is None:
        if not os.path.exists(_REF_PATH):
            raise FileNotFoundError(f"{_REF_PATH} not built (run `make -C oracle ref`)")
        R = ctypes.CDLL(_REF_PATH)
        R.ref_gsek_forward_dd.argtypes = [_i, _i, _i, _d, _d, _d, _d, _d, _d, _d, _d, _i, _dp,
                                          _dp, _dp, _dp, _dp, _dp, _dp]
        R.ref_gsek_forward_dd.restype = _i
        R.ref_gsek_create.argtypes = [_i, _i, _i, _d, _d, _d, _d, _d, _d, _d, _d]
        R.ref_gsek_create.restype = _vp
        R.ref_gsek_eval.argtypes = [_vp, _i, _dp, _dp, _dp, _dp, _dp]
        R.ref_gsek_eval.restype = _i
        R.ref_gsek_destroy.argtypes = [_vp]
        R.ref_gsek_destroy.restype = None
        R.ref_spread.argtypes = [_i, _i, _i, _i, _d, _d, _i, _vp, _d, _d, _d, _i, _vp]
        R.ref_spread.restype = _i
        R.ref_gather.argtypes = [_i, _i, _i, _i, _d, _d, _i, _vp, _d, _d, _d, _vp, _dp, _dp, _dp]
        R.ref_gather.restype = _i
        R.ref_spread_on_grid.argtypes = [_i, _i, _i, _i, _d, _d, _d, _d, _d, _vp, _vp]
        R.ref_spread_on_grid.restype = _i
        R.ref_efield.argtypes = [_i, _i, _i, _i, _d, _d, _d, _vp, _vp, _vp, _vp]
        R.ref_efield.restype = _i
        R.ref_dipole.argtypes = [_i, _i, _i, _i, _d, _d, _d, _vp, _dp]
        R.ref_dipole.restype = _i
        R.ref_green_mul_d.argtypes = [_i, _i, _i, _d, _d, _d, _d, _dp]
        R.ref_green_mul_d.restype = _i
        R.ref_ewald_recip.argtypes = [_d, _i, _d, _d, _d, _d, _i, _dp, _dp, _dp, _dp]
        R.ref_ewald_recip.restype = _d
        R.ref_ewald_direct.argtypes = [_d, _d, _d, _d, _d, _d, _i, _dp, _i, _ip, _ip, _dp, _dp,
                                       _dp]
        R.ref_ewald_direct.restype = _d
        R.ref_grid_save.argtypes = [_i, _i, _i, _i, _vp, ctypes.c_char_p]
        R.ref_grid_save.restype = _i
        _ref = R
    return _ref


# --------------------------------------------------------------------------
# Parameters shared by every reference driver (cpu_gse.cpp:424-426)
# --------------------------------------------------------------------------
def gse_params(sigma: float, kappa: float = 0.4, lambda_sigma1: float = 3.0):
    """sigma1, sigma2, rcut1 exactly as CpuGSE::setParam / CpuGSEk::spreadCharge1
    compute them (CpuGSE.cpp:33-44, CpuGSEk.cpp:30-33)."""
    sigma1 = sigma * np.sqrt(kappa)
    sigma2 = sigma * np.sqrt(1.0 - 2.0 * kappa)
    rcut1 = lambda_sigma1 * np.sqrt(2.0) * sigma1
    return float(sigma1), float(sigma2), float(rcut1)


def _xyzq(xyzq: np.ndarray, dtype) -> np.ndarray:
    a = np.ascontiguousarray(xyzq, dtype=dtype).reshape(-1, 4)
    return a


def spread(M, box, sigma, rcut, xyzq, dtype=np.float64, normalize=False) -> np.ndarray:
    """rho[z, y, x] from CpuGaussCharge::spreadChargeToGrid (restated)."""
    sx, sy, sz = M
    a = _xyzq(xyzq, dtype)
    rho = np.zeros((sz, sy, sx), dtype=dtype)
    sfx, p = ("d", _dp) if dtype == np.float64 else ("f", _fp)
    rc = getattr(lib(), f"orc_spread_{sfx}")(sx, sy, sz, sigma, rcut, a.shape[0], _ptr(a, p),
                                              box[0], box[1], box[2], int(normalize),
                                              _ptr(rho, p))
    if rc:
        raise RuntimeError("orc_spread failed")
    return rho


def gather(M, box, sigma, rcut, xyzq, phi, dtype=np.float64):
    """(fx, fy, fz) from CpuGaussCharge::interpolateForce (restated, no ccelec)."""
    sx, sy, sz = M
    a = _xyzq(xyzq, dtype)
    ph = np.ascontiguousarray(phi, dtype=dtype)
    n = a.shape[0]
    fx, fy, fz = (np.zeros(n) for _ in range(3))
    sfx, p = ("d", _dp) if dtype == np.float64 else ("f", _fp)
    getattr(lib(), f"orc_gather_{sfx}")(sx, sy, sz, sigma, rcut, n, _ptr(a, p), box[0], box[1],
                                        box[2], _ptr(ph, p), _ptr(fx), _ptr(fy), _ptr(fz))
    return fx, fy, fz


def green_mul(M, box, sigma, rhoK: np.ndarray, dtype=np.float64) -> np.ndarray:
    """CpuGreensFuncGSE::mul on a complex half spectrum [z][y][x/2+1] (copy)."""
    sx, sy, sz = M
    k = np.ascontiguousarray(rhoK, dtype=np.complex128 if dtype == np.float64 else np.complex64).copy()
    sfx, p = ("d", _dp) if dtype == np.float64 else ("f", _fp)
    getattr(lib(), f"orc_green_mul_{sfx}")(sx, sy, sz, box[0], box[1], box[2], sigma,
                                           k.ctypes.data_as(p))
    return k


def energy(M, box, rho, phi, ccelec=CCELEC, dtype=np.float64) -> float:
    sx, sy, sz = M
    sfx, p = ("d", _dp) if dtype == np.float64 else ("f", _fp)
    r = np.ascontiguousarray(rho, dtype=dtype)
    f = np.ascontiguousarray(phi, dtype=dtype)
    return float(getattr(lib(), f"orc_energy_{sfx}")(sx, sy, sz, box[0], box[1], box[2], ccelec,
                                                     _ptr(r, p), _ptr(f, p)))


def _grid(a, dtype, M):
    sx, sy, sz = M
    g = np.ascontiguousarray(a, dtype=dtype)
    if g.size != sx * sy * sz:
        raise ValueError("grid size mismatch")
    return g.reshape(sz, sy, sx)


def spread_on_grid(M, box, sigma, rcut, rho, dtype=np.float64) -> np.ndarray:
    """rhoS[z, y, x] from CpuGaussCharge::spreadChargeOnGrid (restated)."""
    sx, sy, sz = M
    r = _grid(rho, dtype, M)
    out = np.zeros_like(r)
    sfx, p = ("d", _dp) if dtype == np.float64 else ("f", _fp)
    rc = getattr(lib(), f"orc_spread_on_grid_{sfx}")(sx, sy, sz, sigma, rcut, box[0], box[1],
                                                     box[2], _ptr(r, p), _ptr(out, p))
    if rc:
        raise RuntimeError("orc_spread_on_grid failed")
    return out


def efield(M, box, phi, dtype=np.float64):
    """(Ex, Ey, Ez)[z, y, x] from CpuGaussCharge::calcElectricFieldOnGrid (restated)."""
    sx, sy, sz = M
    f = _grid(phi, dtype, M)
    E = [np.zeros_like(f) for _ in range(3)]
    sfx, p = ("d", _dp) if dtype == np.float64 else ("f", _fp)
    getattr(lib(), f"orc_efield_{sfx}")(sx, sy, sz, box[0], box[1], box[2], _ptr(f, p),
                                        *(_ptr(e, p) for e in E))
    return tuple(E)


def dipole_sum(M, box, rho, dtype=np.float64) -> np.ndarray:
    """(x, y, z) from CpuGaussCharge::calcDipoleSum (restated)."""
    sx, sy, sz = M
    r = _grid(rho, dtype, M)
    out = np.zeros(3)
    sfx, p = ("d", _dp) if dtype == np.float64 else ("f", _fp)
    getattr(lib(), f"orc_dipole_{sfx}")(sx, sy, sz, box[0], box[1], box[2], _ptr(r, p),
                                        _ptr(out))
    return out


def fft_r2c(x: np.ndarray) -> np.ndarray:
    """FFTW-convention 3-D r2c of a real [nz][ny][nx] array (project FFT)."""
    nz, ny, nx = x.shape
    a = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex128)
    lib().orc_fft_r2c_3d(nx, ny, nz, _ptr(a), out.ctypes.data_as(_dp))
    return out


def fft_c2r(k: np.ndarray, nx: int) -> np.ndarray:
    nz, ny, _ = k.shape
    a = np.ascontiguousarray(k, dtype=np.complex128)
    out = np.zeros((nz, ny, nx), dtype=np.float64)
    lib().orc_fft_c2r_3d(nx, ny, nz, a.ctypes.data_as(_dp), _ptr(out))
    return out


def gsek_forward(M, box, sigma, xyzq, kappa=0.4, lambda_sigma1=3.0, ccelec=CCELEC,
                 want_grids=False):
    """One CpuGSEk<double,double> force evaluation, restated.

    Returns (energy, forces[n,3]) or (energy, forces, rhoS, phi)."""
    sx, sy, sz = M
    a = _xyzq(xyzq, np.float64)
    n = a.shape[0]
    fx, fy, fz = (np.zeros(n) for _ in range(3))
    e = np.zeros(1)
    rho = np.zeros((sz, sy, sx)) if want_grids else None
    phi = np.zeros((sz, sy, sx)) if want_grids else None
    rc = lib().orc_gsek_forward_d(sx, sy, sz, sigma, kappa, lambda_sigma1, box[0], box[1], box[2],
                                  ccelec, n, _ptr(a), _ptr(e), _ptr(fx), _ptr(fy), _ptr(fz),
                                  _ptr(rho), _ptr(phi))
    if rc:
        raise RuntimeError(f"orc_gsek_forward_d failed ({rc})")
    F = np.stack([fx, fy, fz], axis=1)
    if want_grids:
        return float(e[0]), F, rho, phi
    return float(e[0]), F


def ewald_recip(sigma, kcut, box, xyzq, ccelec=CCELEC, forces=True):
    a = _xyzq(xyzq, np.float64)
    n = a.shape[0]
    if forces:
        fx, fy, fz = (np.zeros(n) for _ in range(3))
        e = lib().orc_ewald_recip(sigma, kcut, box[0], box[1], box[2], ccelec, n, _ptr(a),
                                  _ptr(fx), _ptr(fy), _ptr(fz))
        return float(e), np.stack([fx, fy, fz], axis=1)
    e = lib().orc_ewald_recip(sigma, kcut, box[0], box[1], box[2], ccelec, n, _ptr(a),
                              _ptr(None), _ptr(None), _ptr(None))
    return float(e), None


def _excl(iblo14, inb14):
    """(n_iblo14, iblo14, inb14) as int32 arrays for the exclusion arguments."""
    if iblo14 is None:
        return 0, None, None
    ib = np.ascontiguousarray(iblo14, dtype=np.int32)
    nb = np.ascontiguousarray(inb14 if inb14 is not None else [0], dtype=np.int32)
    if len(ib) and len(nb) < ib[-1]:
        raise ValueError("inb14 is shorter than iblo14[-1]")
    return len(ib), ib, nb


def ewald_direct(sigma, rcut, box, xyzq, ccelec=CCELEC, iblo14=None, inb14=None):
    """CpuEwaldDirect::calcForceEnergy restated (gse_oracle.c), with the
    exclusion lists of setupExclusions when iblo14/inb14 are given."""
    a = _xyzq(xyzq, np.float64)
    n = a.shape[0]
    fx, fy, fz = (np.zeros(n) for _ in range(3))
    ne, ib, nb = _excl(iblo14, inb14)
    e = lib().orc_ewald_direct(sigma, rcut, box[0], box[1], box[2], ccelec, n, _ptr(a), ne,
                               _ptr(ib, _ip), _ptr(nb, _ip), _ptr(fx), _ptr(fy), _ptr(fz))
    return float(e), np.stack([fx, fy, fz], axis=1)


def force_rms(F: np.ndarray, Fref: np.ndarray) -> float:
    """Relative force RMS error, Erms of cpu_gse.cpp:131-146."""
    d = np.asarray(F, dtype=np.float64) - np.asarray(Fref, dtype=np.float64)
    return float(np.sqrt(np.sum(d * d) / np.sum(np.asarray(Fref, dtype=np.float64) ** 2)))


# --------------------------------------------------------------------------
# Reference build (oracle/_ref) wrappers
# --------------------------------------------------------------------------
def ref_gsek_forward(M, box, sigma, xyzq, kappa=0.4, lambda_sigma=3.0, lambda_sigma1=3.0,
                     ccelec=CCELEC, want_grids=False):
    sx, sy, sz = M
    a = _xyzq(xyzq, np.float64)
    n = a.shape[0]
    fx, fy, fz = (np.zeros(n) for _ in range(3))
    e = np.zeros(1)
    rho = np.zeros((sz, sy, sx)) if want_grids else None
    phi = np.zeros((sz, sy, sx)) if want_grids else None
    ref().ref_gsek_forward_dd(sx, sy, sz, sigma, kappa, lambda_sigma, lambda_sigma1, box[0], box[1],
                              box[2], ccelec, n, _ptr(a), _ptr(e), _ptr(fx), _ptr(fy), _ptr(fz),
                              _ptr(rho), _ptr(phi))
    F = np.stack([fx, fy, fz], axis=1)
    if want_grids:
        return float(e[0]), F, rho, phi
    return float(e[0]), F


def ref_spread(M, box, sigma, rcut, xyzq, dtype=np.float64, normalize=False):
    sx, sy, sz = M
    a = _xyzq(xyzq, dtype)
    rho = np.zeros((sz, sy, sx), dtype=dtype)
    ref().ref_spread(0 if dtype == np.float64 else 1, sx, sy, sz, sigma, rcut, a.shape[0],
                     a.ctypes.data, box[0], box[1], box[2], int(normalize), rho.ctypes.data)
    return rho


def ref_gather(M, box, sigma, rcut, xyzq, phi, dtype=np.float64):
    sx, sy, sz = M
    a = _xyzq(xyzq, dtype)
    ph = np.ascontiguousarray(phi, dtype=dtype)
    n = a.shape[0]
    fx, fy, fz = (np.zeros(n) for _ in range(3))
    ref().ref_gather(0 if dtype == np.float64 else 1, sx, sy, sz, sigma, rcut, n, a.ctypes.data,
                     box[0], box[1], box[2], ph.ctypes.data, _ptr(fx), _ptr(fy), _ptr(fz))
    return fx, fy, fz


def ref_spread_on_grid(M, box, sigma, rcut, rho, dtype=np.float64):
    sx, sy, sz = M
    r = _grid(rho, dtype, M)
    out = np.zeros_like(r)
    ref().ref_spread_on_grid(0 if dtype == np.float64 else 1, sx, sy, sz, sigma, rcut, box[0],
                             box[1], box[2], r.ctypes.data, out.ctypes.data)
    return out


def ref_efield(M, box, phi, dtype=np.float64):
    sx, sy, sz = M
    f = _grid(phi, dtype, M)
    E = [np.zeros_like(f) for _ in range(3)]
    ref().ref_efield(0 if dtype == np.float64 else 1, sx, sy, sz, box[0], box[1], box[2],
                     f.ctypes.data, *(e.ctypes.data for e in E))
    return tuple(E)


def ref_dipole_sum(M, box, rho, dtype=np.float64):
    sx, sy, sz = M
    r = _grid(rho, dtype, M)
    out = np.zeros(3)
    ref().ref_dipole(0 if dtype == np.float64 else 1, sx, sy, sz, box[0], box[1], box[2],
                     r.ctypes.data, _ptr(out))
    return out


def ref_green_mul(M, box, sigma, rhoK):
    sx, sy, sz = M
    k = np.ascontiguousarray(rhoK, dtype=np.complex128).copy()
    ref().ref_green_mul_d(sx, sy, sz, box[0], box[1], box[2], sigma, k.ctypes.data_as(_dp))
    return k


def ref_ewald_recip(sigma, kcut, box, xyzq, ccelec=CCELEC):
    a = _xyzq(xyzq, np.float64)
    n = a.shape[0]
    fx, fy, fz = (np.zeros(n) for _ in range(3))
    e = ref().ref_ewald_recip(sigma, kcut, box[0], box[1], box[2], ccelec, n, _ptr(a), _ptr(fx),
                              _ptr(fy), _ptr(fz))
    return float(e), np.stack([fx, fy, fz], axis=1)


def ref_ewald_direct(sigma, rcut, box, xyzq, ccelec=CCELEC, iblo14=None, inb14=None):
    a = _xyzq(xyzq, np.float64)
    n = a.shape[0]
    fx, fy, fz = (np.zeros(n) for _ in range(3))
    ne, ib, nb = _excl(iblo14, inb14)
    e = ref().ref_ewald_direct(sigma, rcut, box[0], box[1], box[2], ccelec, n, _ptr(a), ne,
                               _ptr(ib, _ip), _ptr(nb, _ip), _ptr(fx), _ptr(fy), _ptr(fz))
    return float(e), np.stack([fx, fy, fz], axis=1)


def ref_grid_save(grid: np.ndarray, filename) -> None:
    """The reference's CpuGrid<T>::save (CpuGrid.h:76-90) of a [z][y][x]
    float64 or float32 grid into `filename`."""
    g = np.ascontiguousarray(grid)
    if g.dtype not in (np.float64, np.float32) or g.ndim != 3:
        raise ValueError("a 3-D float64 or float32 grid")
    sz, sy, sx = g.shape
    ref().ref_grid_save(0 if g.dtype == np.float64 else 1, sx, sy, sz, g.ctypes.data,
                        os.fsencode(str(filename)))
