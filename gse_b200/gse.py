"""Python mirror of the reference's GSE-k class API, running on the B200.

Class and method names, argument order and meaning follow ap-hynninen/GSE:

  CpuGrid<T>            Grid.h:12-55, CpuGrid.h:17-108  (host container)
  CpuGaussCharge<AT,CT> CpuGaussCharge.h:11-49
  CpuGreensFuncGSE<T>   CpuGreensFuncGSE.h:10-19
  CpuFFTSolver<T>       CpuFFTSolver.h:12-42
  CpuGSE<AT,CT>/CpuGSEk CpuGSE.h:19-68, CpuGSEk.h:19-37
  CpuEwaldRecip         CpuEwaldRecip.h:11-44 (calcForceEnergy; FP64)
  CpuEwaldDirect        CpuEwaldDirect.h:10-44 (FP64)
  Erms, loadArray, saveForce, readForce   cpu_gse.cpp:128-196 (text I/O)

The template parameters become a ``precision`` argument: "fp64" is
<double,double>; "mixed" is <double,float> (FP32 xyzq and grids, double
forces and energies).  Where the reference asserts or exits, these classes
raise GseError.  Every computation runs in libgse_b200.so on the GPU; there is
no CPU fallback.

Arrays: xyzq is an (n, 4) array of the calculation type (numpy on the host,
or a CUDA torch tensor); forceX/Y/Z are float64 arrays of length n written in
place (numpy or CUDA torch tensors).
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from ._lib import GseError, check, ptr, ptr_f64, ptr_records

CCELEC = 332.0716


def _ct(precision: str):
    if precision not in _lib.PRECISION:
        raise GseError(1, f"unknown precision {precision!r} (use 'fp64' or 'mixed')")
    return np.float64 if precision == "fp64" else np.float32


class Context:
    """Owner of one gse_context_t (grids, FFT plans, staging buffers)."""

    def __init__(self, sizeX, sizeY, sizeZ, sigma=1.0, kappa=0.4, lambdaSigma=3.0,
                 lambdaSigma1=3.0, boxx=1.0, boxy=1.0, boxz=1.0, ccelec=CCELEC,
                 precision="fp64", device=0):
        L = _lib.load()
        p = _lib.gse_params_t()
        L.gse_params_default(ctypes.byref(p))
        p.size_x, p.size_y, p.size_z = int(sizeX), int(sizeY), int(sizeZ)
        p.sigma, p.kappa = float(sigma), float(kappa)
        p.lambda_sigma, p.lambda_sigma1 = float(lambdaSigma), float(lambdaSigma1)
        p.box_x, p.box_y, p.box_z = float(boxx), float(boxy), float(boxz)
        p.ccelec = float(ccelec)
        _ct(precision)
        p.precision = _lib.PRECISION[precision]
        p.device = int(device)
        h = ctypes.c_void_p()
        check(L.gse_create(ctypes.byref(p), ctypes.byref(h)))
        self._L = L
        self.h = h
        self.params = p
        self.precision = precision
        self.dtype = _ct(precision)
        self.shape = (int(sizeZ), int(sizeY), int(sizeX))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self._L.gse_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _xyzq(self, xyzq, n):
        return ptr_records(xyzq, int(n), np.dtype(self.dtype).itemsize)

    # -- thin wrappers of the C ABI ---------------------------------------
    def set_stream(self, stream_handle: int):
        check(self._L.gse_set_stream(self.h, stream_handle))

    def set_box(self, bx, by, bz):
        check(self._L.gse_set_box(self.h, bx, by, bz))

    def synchronize(self):
        check(self._L.gse_synchronize(self.h))

    def spread_charge(self, n, xyzq):
        check(self._L.gse_spread_charge(self.h, int(n), self._xyzq(xyzq, n)))

    def solve_poisson(self):
        check(self._L.gse_solve_poisson(self.h))

    def calculate_energy(self, out=None) -> float:
        if out is not None:
            check(self._L.gse_calculate_energy(self.h, ptr(out)))
            return None
        e = ctypes.c_double()
        check(self._L.gse_calculate_energy(self.h, ctypes.addressof(e)))
        return e.value

    def interpolate_force(self, n, xyzq, fx, fy, fz):
        n = int(n)
        check(self._L.gse_interpolate_force(self.h, n, self._xyzq(xyzq, n),
                                            ptr_f64(fx, n, "fx"), ptr_f64(fy, n, "fy"),
                                            ptr_f64(fz, n, "fz")))

    def forward(self, n, xyzq, fx=None, fy=None, fz=None, energy_out=None) -> Optional[float]:
        n = int(n)
        f = [ptr_f64(a, n, k) for a, k in ((fx, "fx"), (fy, "fy"), (fz, "fz"))]
        if energy_out is not None:
            check(self._L.gse_forward(self.h, n, self._xyzq(xyzq, n),
                                      ptr_f64(energy_out, 1, "energy_out"), *f))
            return None
        e = ctypes.c_double()
        check(self._L.gse_forward(self.h, n, self._xyzq(xyzq, n), ctypes.addressof(e), *f))
        return e.value

    def get_grid(self, which, out=None):
        if out is None:
            out = np.empty(self.shape, dtype=self.dtype)
        check(self._L.gse_get_grid(self.h, int(which), ptr(out)))
        return out

    def set_grid(self, which, data):
        a = data
        if isinstance(data, np.ndarray):
            a = np.ascontiguousarray(data, dtype=self.dtype)
        check(self._L.gse_set_grid(self.h, int(which), ptr(a)))

    def gauss_spread(self, sigma, rcut, n, xyzq, boxx, boxy, boxz, normalize, rho_out):
        check(self._L.gse_gauss_spread(self.h, sigma, rcut, int(n), self._xyzq(xyzq, n), boxx,
                                       boxy, boxz, int(bool(normalize)), ptr(rho_out)))

    def gauss_interpolate(self, sigma, rcut, n, xyzq, boxx, boxy, boxz, phi, fx, fy, fz):
        n = int(n)
        check(self._L.gse_gauss_interpolate(self.h, sigma, rcut, n, self._xyzq(xyzq, n), boxx,
                                            boxy, boxz, ptr(phi), ptr_f64(fx, n, "fx"),
                                            ptr_f64(fy, n, "fy"), ptr_f64(fz, n, "fz")))

    def green_mul(self, sigma, boxx, boxy, boxz, rho_k):
        check(self._L.gse_green_mul(self.h, sigma, boxx, boxy, boxz, ptr(rho_k)))

    def fft_solve(self, sigma, boxx, boxy, boxz, rho, phi):
        check(self._L.gse_fft_solve(self.h, sigma, boxx, boxy, boxz, ptr(rho), ptr(phi)))

    def interpolate_field(self, n, xyzq, ex, ey, ez):
        """Electric field at the atoms (force per unit charge) from phiM."""
        n = int(n)
        check(self._L.gse_interpolate_field(self.h, n, self._xyzq(xyzq, n),
                                            ptr_f64(ex, n, "ex"), ptr_f64(ey, n, "ey"),
                                            ptr_f64(ez, n, "ez")))

    def virial(self, out=None):
        """Reciprocal-space virial (xx, yy, zz, xy, xz, yz) of the current rhoS."""
        if out is None:
            v = np.zeros(6)
            check(self._L.gse_virial(self.h, ptr(v)))
            return v
        check(self._L.gse_virial(self.h, ptr(out)))
        return out

    def gauss_spread_on_grid(self, sigma, rcut, boxx, boxy, boxz, rho, rho_s):
        check(self._L.gse_gauss_spread_on_grid(self.h, sigma, rcut, boxx, boxy, boxz, ptr(rho),
                                               ptr(rho_s)))

    def gauss_efield_on_grid(self, boxx, boxy, boxz, phi, ex, ey, ez):
        check(self._L.gse_gauss_efield_on_grid(self.h, boxx, boxy, boxz, ptr(phi), ptr(ex),
                                               ptr(ey), ptr(ez)))

    def gauss_dipole_sum(self, boxx, boxy, boxz, rho, dip):
        check(self._L.gse_gauss_dipole_sum(self.h, boxx, boxy, boxz, ptr(rho), ptr(dip)))

    def adjoint(self, n, xyzq, dLdE, gfx, gfy, gfz, dq, dx, dy, dz):
        """dL/dq and dL/dx for dL/dE = dLdE and dL/dF = (gfx, gfy, gfz) (may be None)."""
        n = int(n)
        g = [ptr_f64(v, n, k) for v, k in ((gfx, "gfx"), (gfy, "gfy"), (gfz, "gfz"))]
        o = [ptr_f64(v, n, k) for v, k in ((dq, "dq"), (dx, "dx"), (dy, "dy"), (dz, "dz"))]
        check(self._L.gse_adjoint(self.h, n, self._xyzq(xyzq, n), float(dLdE), *g, *o))

    def paths(self) -> int:
        """Bits of the implementation paths taken (_lib.PATH_*)."""
        f = ctypes.c_int()
        check(self._L.gse_get_paths(self.h, ctypes.byref(f)))
        return f.value

    def set_timing(self, enable: bool):
        check(self._L.gse_set_timing(self.h, int(bool(enable))))

    def launch_count(self) -> int:
        c = ctypes.c_longlong()
        check(self._L.gse_get_launch_count(self.h, ctypes.addressof(c)))
        return c.value

    def get_timing(self, reset: bool = False):
        """{stage: (total_ms, launches)} of the device stage timers."""
        ms = np.zeros(len(_lib.STAGES), dtype=np.float64)
        cnt = np.zeros(len(_lib.STAGES), dtype=np.int64)
        check(self._L.gse_get_timing(self.h, ms.ctypes.data, cnt.ctypes.data, int(bool(reset))))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_lib.STAGES)}


def _xyzq_arg(xyzq, dtype):
    if isinstance(xyzq, np.ndarray):
        a = np.ascontiguousarray(xyzq, dtype=dtype)
        if a.ndim != 2 or a.shape[1] != 4:
            a = a.reshape(-1, 4)
        return a
    return xyzq  # device tensor: caller guarantees dtype/layout


# ---------------------------------------------------------------------------
# Reference API mirror
# ---------------------------------------------------------------------------
class CpuGrid:
    """Host grid of sizeX x sizeY x sizeZ values, x fastest (CpuGrid.h:17-108)."""

    def __init__(self, sizeX, sizeY, sizeZ, dtype=np.float64):
        self.sizeX, self.sizeY, self.sizeZ = int(sizeX), int(sizeY), int(sizeZ)
        self.size = self.sizeX * self.sizeY * self.sizeZ
        self.data = np.zeros((self.sizeZ, self.sizeY, self.sizeX), dtype=dtype)

    def getDataPointer(self):
        return self.data

    def getSizeX(self):
        return self.sizeX

    def getSizeY(self):
        return self.sizeY

    def getSizeZ(self):
        return self.sizeZ

    def getSize(self):
        return self.size

    def getPos(self, x, y, z):
        return (x % self.sizeX) + ((y % self.sizeY) + (z % self.sizeZ) * self.sizeY) * self.sizeX

    def clear(self):
        self.data[...] = 0

    def add(self, other):
        self.data += other.data

    def sub(self, other):
        self.data -= other.data.astype(self.data.dtype)

    def copy(self, other):
        self.data[...] = other.data.astype(self.data.dtype)

    def scale(self, val):
        self.data *= val

    def sum(self):
        return self.data.sum()

    def maxAbsValue(self):
        return np.abs(self.data).max()

    def getDataValue(self, x, y, z):
        return self.data[z % self.sizeZ, y % self.sizeY, x % self.sizeX]

    def save(self, filename):
        """One value per line, z outermost (CpuGrid.h:76-106)."""
        with open(filename, "w") as f:
            for v in self.data.reshape(-1):
                f.write(f"{v:g}\n")


def Erms(n, refx, refy, refz, x, y, z) -> float:
    """Relative RMS difference of two force sets, sqrt(sum |F - Fref|^2 / sum
    |Fref|^2) (cpu_gse.cpp:128-145)."""
    r = np.stack([np.asarray(v, np.float64)[:n] for v in (refx, refy, refz)])
    d = np.stack([np.asarray(v, np.float64)[:n] for v in (x, y, z)]) - r
    return float(np.sqrt((d * d).sum() / (r * r).sum()))


def loadArray(width, numLine, filename, dtype=np.float64) -> np.ndarray:
    """numLine records of `width` whitespace-separated values
    (cpu_gse.cpp:150-170), as an array [numLine, width]; GseError where the
    reference exits on a short or unreadable file."""
    try:
        with open(filename) as f:
            tok = f.read().split()
    except OSError as e:
        raise GseError(1, f"cannot open {filename}: {e}") from None
    if len(tok) < width * numLine:
        raise GseError(1, f"error reading {filename}")
    conv = int if np.issubdtype(np.dtype(dtype), np.integer) else float
    return np.array([conv(t) for t in tok[:width * numLine]], dtype=dtype).reshape(numLine, width)


def saveForce(filename, numCoord, forceX, forceY, forceZ):
    """'fx fy fz' per line in the iostream default format, six significant
    digits (cpu_gse.cpp:172-182)."""
    with open(filename, "w") as f:
        for i in range(numCoord):
            f.write(f"{forceX[i]:g} {forceY[i]:g} {forceZ[i]:g}\n")


def readForce(filename, numCoord, dtype=np.float64):
    """The file saveForce writes (cpu_gse.cpp:185-196): (fx, fy, fz)."""
    a = loadArray(3, numCoord, filename, dtype)
    return a[:, 0].copy(), a[:, 1].copy(), a[:, 2].copy()


class CpuGaussCharge:
    """CpuGaussCharge<AT,CT> (CpuGaussCharge.h:11-49) on the GPU."""

    def __init__(self, sizeX, sizeY, sizeZ, precision="fp64", device=0):
        self.sizeX, self.sizeY, self.sizeZ = int(sizeX), int(sizeY), int(sizeZ)
        self.precision = precision
        self.dtype = _ct(precision)
        # the stage calls carry their own sigma, rcut and box; the context's
        # own parameters only need to describe a valid stencil
        self._ctx = Context(sizeX, sizeY, sizeZ, sigma=1.0, boxx=sizeX, boxy=sizeY, boxz=sizeZ,
                            precision=precision, device=device)

    def _check(self, grid: CpuGrid):
        if (grid.sizeX, grid.sizeY, grid.sizeZ) != (self.sizeX, self.sizeY, self.sizeZ):
            raise GseError(1, "grid size mismatch (CpuGaussCharge.cpp:240-242)")

    def spreadChargeToGrid(self, sigma, rcut, numCoord, xyzq, boxx, boxy, boxz, rho: CpuGrid,
                           normalize=False):
        self._check(rho)
        if rho.data.dtype != self.dtype:
            raise GseError(1, "rho grid dtype does not match precision")
        self._ctx.gauss_spread(sigma, rcut, numCoord, _xyzq_arg(xyzq, self.dtype), boxx, boxy,
                               boxz, normalize, rho.data)

    def interpolateForce(self, sigma, rcut, numCoord, xyzq, boxx, boxy, boxz, phi: CpuGrid,
                         forceX, forceY, forceZ):
        self._check(phi)
        ph = np.ascontiguousarray(phi.data, dtype=self.dtype)
        self._ctx.gauss_interpolate(sigma, rcut, numCoord, _xyzq_arg(xyzq, self.dtype), boxx,
                                    boxy, boxz, ph, forceX, forceY, forceZ)

    def _grid_arg(self, grid: CpuGrid):
        self._check(grid)
        if grid.data.dtype != self.dtype:
            raise GseError(1, "grid dtype does not match precision")
        return grid.data

    def spreadChargeOnGrid(self, sigma, rcut, boxx, boxy, boxz, rho: CpuGrid, rhoS: CpuGrid):
        """On-grid Gaussian convolution (CpuGaussCharge.cpp:390-519)."""
        self._ctx.gauss_spread_on_grid(sigma, rcut, boxx, boxy, boxz, self._grid_arg(rho),
                                       self._grid_arg(rhoS))

    def calcElectricFieldOnGrid(self, boxx, boxy, boxz, phi: CpuGrid, Ex: CpuGrid, Ey: CpuGrid,
                                Ez: CpuGrid):
        """Forward-difference field on the grid (CpuGaussCharge.cpp:62-98)."""
        self._ctx.gauss_efield_on_grid(boxx, boxy, boxz, self._grid_arg(phi), self._grid_arg(Ex),
                                       self._grid_arg(Ey), self._grid_arg(Ez))

    def calcDipoleSum(self, boxx, boxy, boxz, rho: CpuGrid):
        """(dipSumX, dipSumY, dipSumZ) of a charge grid (CpuGaussCharge.cpp:188-226); the
        reference returns them through reference arguments."""
        dip = np.zeros(3)
        self._ctx.gauss_dipole_sum(boxx, boxy, boxz, self._grid_arg(rho), dip)
        return float(dip[0]), float(dip[1]), float(dip[2])

    def calcSupportSize(self, rcut, boxx, boxy, boxz):
        """Number of offsets with r^2 < rcut^2 (CpuGaussCharge.cpp:28-56): the
        spacings and rcut^2 rounded to the calculation type, the distances
        formed and summed in it, in the reference's order."""
        ct = np.dtype(getattr(self, "dtype", np.float64)).type
        hd = [boxx / self.sizeX, boxy / self.sizeY, boxz / self.sizeZ]
        n = [int(np.ceil(rcut / v)) for v in hd]
        t = [(np.abs(np.arange(-k, k + 1)) - 1).astype(ct) * ct(v) for k, v in zip(n, hd)]
        dx, dy, dz = t[0][None, None, :], t[1][None, :, None], t[2][:, None, None]
        r2 = (dx * dx + dy * dy) + dz * dz
        return int(np.count_nonzero(r2 < ct(rcut * rcut)))


class CpuGreensFunc:
    """Base class (CpuGreensFunc.h:10-19)."""

    def mul(self, nfftX, nfftY, nfftZ, boxx, boxy, boxz, sigma, rho):
        raise NotImplementedError


class CpuGreensFuncGSE(CpuGreensFunc):
    """CpuGreensFuncGSE<T>::mul (CpuGreensFuncGSE.cpp:9-57) on the GPU.

    ``rho`` is the k-space grid, a CpuGrid of ((nfftX/2+1)*2, nfftY, nfftZ)
    reals holding interleaved complex values."""

    def __init__(self, precision="fp64", device=0):
        self.precision = precision
        self.device = device
        self._ctx = None

    def _context(self, nx, ny, nz):
        if self._ctx is None or self._ctx.shape != (nz, ny, nx):
            self._ctx = Context(nx, ny, nz, boxx=nx, boxy=ny, boxz=nz, precision=self.precision,
                                device=self.device)
        return self._ctx

    def mul(self, nfftX, nfftY, nfftZ, boxx, boxy, boxz, sigma, rho: CpuGrid):
        if (nfftX // 2 + 1) * 2 != rho.sizeX or nfftY != rho.sizeY or nfftZ != rho.sizeZ:
            raise GseError(1, "k-space grid size mismatch (CpuGreensFuncGSE.cpp:13-15)")
        ctx = self._context(nfftX, nfftY, nfftZ)
        if rho.data.dtype != ctx.dtype:
            raise GseError(1, "k-space grid dtype does not match precision")
        ctx.green_mul(sigma, boxx, boxy, boxz, rho.data)


class CpuFFTSolver:
    """CpuFFTSolver<T> (CpuFFTSolver.h:12-42): phi = c2r(G r2c(rho))."""

    def __init__(self, greensFunc: CpuGreensFuncGSE, sizeX, sizeY, sizeZ):
        if not isinstance(greensFunc, CpuGreensFuncGSE):
            raise GseError(7, "only the GSE Green's function is implemented on the GPU")
        self.greensFunc = greensFunc
        self.sizeX, self.sizeY, self.sizeZ = int(sizeX), int(sizeY), int(sizeZ)
        self._ctx = Context(sizeX, sizeY, sizeZ, boxx=sizeX, boxy=sizeY, boxz=sizeZ,
                            precision=greensFunc.precision, device=greensFunc.device)

    def run(self, phi: CpuGrid, rho: CpuGrid, sigma, boxx, boxy, boxz):
        for g in (phi, rho):
            if (g.sizeX, g.sizeY, g.sizeZ) != (self.sizeX, self.sizeY, self.sizeZ):
                raise GseError(1, "grid size mismatch (CpuFFTSolver.cpp:78-83)")
        r = np.ascontiguousarray(rho.data, dtype=self._ctx.dtype)
        self._ctx.fft_solve(sigma, boxx, boxy, boxz, r, phi.data)


class CpuGSE:
    """Common base of the GSE drivers (CpuGSE.h:19-68)."""

    def __init__(self, sizeX, sizeY, sizeZ, sigma, kappa, lambdaSigma, lambdaSigma1, boxx, boxy,
                 boxz, ccelec=CCELEC, precision="fp64", device=0):
        if not (0.0 <= kappa <= 0.5):
            raise GseError(1, "kappa must lie in [0, 0.5] (CpuGSE.cpp:35-36)")
        self.ccelec = ccelec
        self.sigma, self.kappa = sigma, kappa
        self.lambdaSigma, self.lambdaSigma1 = lambdaSigma, lambdaSigma1
        self.sigma1 = sigma * np.sqrt(kappa)
        self.sigma2 = sigma * np.sqrt(1.0 - 2.0 * kappa)
        self.boxx, self.boxy, self.boxz = boxx, boxy, boxz
        self.precision = precision
        self.dtype = _ct(precision)
        self._ctx = Context(sizeX, sizeY, sizeZ, sigma, kappa, lambdaSigma, lambdaSigma1, boxx,
                            boxy, boxz, ccelec, precision, device)
        self.rhoS = CpuGrid(sizeX, sizeY, sizeZ, self.dtype)
        self.phiM = CpuGrid(sizeX, sizeY, sizeZ, self.dtype)

    def printInfo(self):
        g = self.rhoS
        print(f"sizeX={g.sizeX} sizeY={g.sizeY} sizeZ={g.sizeZ}")
        print(f"sigma={self.sigma} sigma1={self.sigma1} sigma2={self.sigma2} kappa={self.kappa}")
        print(f"lambdaSigma1={self.lambdaSigma1} lambdaSigma={self.lambdaSigma}")

    def setBoxSize(self, boxx, boxy, boxz):
        self._ctx.set_box(boxx, boxy, boxz)
        self.boxx, self.boxy, self.boxz = boxx, boxy, boxz

    def interpolateForce(self, numCoord, xyzq, forceX, forceY, forceZ):
        self._ctx.interpolate_force(numCoord, _xyzq_arg(xyzq, self.dtype), forceX, forceY, forceZ)

    def getRhoS(self) -> CpuGrid:
        self._ctx.get_grid(_lib.GRID_RHO, self.rhoS.data)
        return self.rhoS

    def getPhi(self) -> CpuGrid:
        self._ctx.get_grid(_lib.GRID_PHI, self.phiM.data)
        return self.phiM

    def interpolateField(self, numCoord, xyzq, fieldX, fieldY, fieldZ):
        """Electric field at the atoms (force per unit charge) from phiM."""
        self._ctx.interpolate_field(numCoord, _xyzq_arg(xyzq, self.dtype), fieldX, fieldY, fieldZ)

    def calculateVirial(self):
        """Reciprocal-space virial (xx, yy, zz, xy, xz, yz) of the current rhoS; the
        reference classes compute none."""
        return self._ctx.virial()

    def getSigma1(self):
        return self.sigma1

    def getSigma2(self):
        return self.sigma2

    def getLambdaSigma1(self):
        return self.lambdaSigma1

    @property
    def context(self) -> Context:
        return self._ctx


class CpuGSEk(CpuGSE):
    """CpuGSEk<AT,CT> (CpuGSEk.h:19-37, CpuGSEk.cpp:30-58) on the GPU."""

    def spreadCharge1(self, numCoord, xyzq):
        self._ctx.spread_charge(numCoord, _xyzq_arg(xyzq, self.dtype))

    def solvePoisson(self):
        self._ctx.solve_poisson()

    def calculateEnergy(self) -> float:
        return self._ctx.calculate_energy()

    def forward(self, numCoord, xyzq, forceX=None, forceY=None, forceZ=None) -> float:
        """spreadCharge1 + solvePoisson + calculateEnergy + interpolateForce in one call."""
        return self._ctx.forward(numCoord, _xyzq_arg(xyzq, self.dtype), forceX, forceY, forceZ)


def ewald_recip(sigma, kcut, box, xyzq, ccelec=CCELEC, forces=True, device=0, stream=None):
    """FP64 Ewald reciprocal sum on the GPU (CpuEwaldRecip::calcForceEnergy,
    CpuEwaldRecip.cpp:87-147).  Returns (E, F[n, 3]) or (E, None)."""
    L = _lib.load()
    a = np.ascontiguousarray(xyzq, dtype=np.float64).reshape(-1, 4)
    n = a.shape[0]
    e = ctypes.c_double()
    if forces:
        f = np.zeros((3, n))
        check(L.gse_ewald_recip(device, stream, sigma, int(kcut), box[0], box[1], box[2], ccelec,
                                n, a.ctypes.data, ctypes.addressof(e), f[0].ctypes.data,
                                f[1].ctypes.data, f[2].ctypes.data))
        return e.value, f.T.copy()
    check(L.gse_ewald_recip(device, stream, sigma, int(kcut), box[0], box[1], box[2], ccelec, n,
                            a.ctypes.data, ctypes.addressof(e), None, None, None))
    return e.value, None


def ewald_direct(sigma, rcut, box, xyzq, iblo14=None, inb14=None, ccelec=CCELEC, forces=True,
                 device=0, stream=None):
    """FP64 Ewald direct sum with self energy on the GPU (CpuEwaldDirect::
    calcForceEnergy, CpuEwaldDirect.cpp:45-131), with the exclusion lists of
    setupExclusions (CpuEwaldDirect.cpp:31-40) when iblo14 and inb14 are given.
    Returns (E, F[n, 3]) or (E, None); F is the gradient dE/dx, as the
    reference's force arrays hold it."""
    L = _lib.load()
    a = np.ascontiguousarray(xyzq, dtype=np.float64).reshape(-1, 4)
    n = a.shape[0]
    nib, ib, nb = 0, None, None
    if iblo14 is not None:
        ib = np.ascontiguousarray(iblo14, dtype=np.int32)
        nb = np.ascontiguousarray(inb14 if inb14 is not None else [], dtype=np.int32)
        nib = ib.shape[0]
        if nib and nb.shape[0] < ib[-1]:
            raise ValueError("inb14 is shorter than iblo14[-1]")
    e = ctypes.c_double()
    f = np.zeros((3, n)) if forces else None
    fp = [f[k].ctypes.data for k in range(3)] if forces else [None] * 3
    check(L.gse_ewald_direct(device, stream, sigma, rcut, box[0], box[1], box[2], ccelec, n,
                             a.ctypes.data, nib, None if ib is None else ib.ctypes.data,
                             None if nb is None else nb.ctypes.data, ctypes.addressof(e), *fp))
    return e.value, (f.T.copy() if forces else None)


class CpuEwaldRecip:
    """CpuEwaldRecip (CpuEwaldRecip.h:11-44) on the GPU in FP64:
    calcForceEnergy(n, xyzq, fx, fy, fz) -> energy, writing the force arrays."""

    def __init__(self, sigma, kcut, boxx, boxy, boxz, ccelec=CCELEC, device=0):
        self.sigma, self.kcut, self.ccelec, self.device = float(sigma), int(kcut), ccelec, device
        self.box = (float(boxx), float(boxy), float(boxz))

    def setSigma(self, sigma):
        self.sigma = float(sigma)

    def setBoxsize(self, boxx, boxy, boxz):
        self.box = (float(boxx), float(boxy), float(boxz))

    def calcForceEnergy(self, n, xyzq, fx, fy, fz) -> float:
        a = np.ascontiguousarray(xyzq, dtype=np.float64).reshape(-1, 4)[:n]
        e, f = ewald_recip(self.sigma, self.kcut, self.box, a, self.ccelec, True, self.device)
        fx[:n], fy[:n], fz[:n] = f[:, 0], f[:, 1], f[:, 2]
        return e


class CpuEwaldDirect:
    """CpuEwaldDirect (CpuEwaldDirect.h:10-44) on the GPU in FP64:
    setupExclusions(n_iblo14, iblo14, inb14), then calcForceEnergy(n, xyzq,
    fx, fy, fz) -> energy including the self energy, writing the gradient
    into the force arrays."""

    def __init__(self, sigma, rcut, boxx, boxy, boxz, ccelec=CCELEC, device=0):
        self.sigma, self.rcut, self.ccelec, self.device = float(sigma), float(rcut), ccelec, device
        self.box = (float(boxx), float(boxy), float(boxz))
        self._iblo14 = self._inb14 = None

    def setupExclusions(self, n_iblo14, iblo14, inb14):
        ib = np.array(iblo14[:n_iblo14], dtype=np.int32)
        self._iblo14 = ib
        self._inb14 = np.array(inb14[:ib[-1] if n_iblo14 else 0], dtype=np.int32)

    def calcForceEnergy(self, n, xyzq, fx, fy, fz) -> float:
        a = np.ascontiguousarray(xyzq, dtype=np.float64).reshape(-1, 4)[:n]
        e, f = ewald_direct(self.sigma, self.rcut, self.box, a, self._iblo14, self._inb14,
                            self.ccelec, True, self.device)
        fx[:n], fy[:n], fz[:n] = f[:, 0], f[:, 1], f[:, 2]
        return e


def ewald_kcut(sigma, box, tol=1e-12):
    """Smallest integer k cut-off with exp(-sigma^2 k^2 / 2) below tol along the longest box side."""
    import math
    kmax = math.sqrt(2.0 * math.log(1.0 / tol)) / sigma
    return int(math.ceil(kmax * max(box) / (2.0 * math.pi)))


class Batch:
    """Many independent GSE-k systems of uneven size evaluated together (mixed
    form).  ``systems`` is a list of dicts with keys size (Mx, My, Mz), box
    (Lx, Ly, Lz) and n.  Atoms are numbered system after system.

    forward(xyzq) -> (energies[S], forces[n_total, 3]); adjoint(...) gives the
    reverse pass; capture()/launch() replay one evaluation from a CUDA graph on
    the batch's own device buffers (``buffers()``); autotune() picks the
    persistent-CTA counts and work order, cached in a text file."""

    def __init__(self, systems, sigma=1.0, kappa=0.4, lambdaSigma1=3.0, ccelec=CCELEC, device=0):
        L = _lib.load()
        p = _lib.gse_params_t()
        L.gse_params_default(ctypes.byref(p))
        p.sigma, p.kappa = float(sigma), float(kappa)
        p.lambda_sigma = p.lambda_sigma1 = float(lambdaSigma1)
        p.ccelec = float(ccelec)
        p.precision = _lib.PRECISION["mixed"]
        p.device = int(device)
        arr = (_lib.gse_system_t * len(systems))()
        for k, s in enumerate(systems):
            arr[k].size_x, arr[k].size_y, arr[k].size_z = (int(v) for v in s["size"])
            arr[k].box_x, arr[k].box_y, arr[k].box_z = (float(v) for v in s["box"])
            arr[k].n = int(s["n"])
        h = ctypes.c_void_p()
        check(L.gse_batch_create(ctypes.byref(p), len(systems), arr, ctypes.byref(h)))
        self._L = L
        self.h = h
        self.systems = list(systems)
        self.counts = [int(s["n"]) for s in systems]
        self.first = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        self.n_total = int(self.first[-1])

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self._L.gse_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> "_lib.gse_batch_info_t":
        i = _lib.gse_batch_info_t()
        check(self._L.gse_batch_info(self.h, ctypes.byref(i)))
        return i

    def set_stream(self, stream_handle: int):
        check(self._L.gse_batch_set_stream(self.h, stream_handle))

    def forward(self, xyzq, energies=None, fx=None, fy=None, fz=None):
        """xyzq: (n_total, 4) float32 host array or CUDA tensor.  Without
        output arguments, returns (energies, forces) as numpy arrays."""
        x = _xyzq_arg(xyzq, np.float32)
        if energies is None and fx is None:
            e = np.zeros(len(self.counts))
            f = np.zeros((3, self.n_total))
            check(self._L.gse_batch_forward(self.h, ptr(x), e.ctypes.data, f[0].ctypes.data,
                                            f[1].ctypes.data, f[2].ctypes.data))
            return e, f.T.copy()
        check(self._L.gse_batch_forward(self.h, ptr(x), ptr(energies), ptr(fx), ptr(fy), ptr(fz)))
        return None

    def adjoint(self, xyzq, dLdE=None, gforces=None):
        """Reverse pass of L(E, F).  dLdE: (S,) ; gforces: (n_total, 3) or None.
        Returns (dL/dq[n], dL/dx[n, 3]) as numpy arrays."""
        x = _xyzq_arg(xyzq, np.float32)
        d = None if dLdE is None else np.ascontiguousarray(dLdE, dtype=np.float64)
        g = None
        if gforces is not None:
            g = np.ascontiguousarray(np.asarray(gforces, dtype=np.float64).T)
        out = np.zeros((4, self.n_total))
        check(self._L.gse_batch_adjoint(
            self.h, ptr(x), None if d is None else d.ctypes.data,
            None if g is None else g[0].ctypes.data, None if g is None else g[1].ctypes.data,
            None if g is None else g[2].ctypes.data, out[0].ctypes.data, out[1].ctypes.data,
            out[2].ctypes.data, out[3].ctypes.data))
        return out[0].copy(), out[1:].T.copy()

    def capture(self, with_adjoint=False):
        check(self._L.gse_batch_capture(self.h, 1 if with_adjoint else 0))

    def launch(self):
        check(self._L.gse_batch_launch(self.h))

    def autotune(self, cache_path=None, use_cache=True):
        check(self._L.gse_batch_autotune(
            self.h, None if cache_path is None else str(cache_path).encode(), 1 if use_cache else 0))

    def set_schedule(self, fused, gather_lanes=16, largest_first=False, scatter_ctas=296,
                     gather_ctas=296):
        """Pin the launch schedule (gse_batch_set_schedule): fused=True runs each
        direction as one persistent cooperative kernel."""
        check(self._L.gse_batch_set_schedule(self.h, int(bool(fused)), int(gather_lanes),
                                             int(bool(largest_first)), int(scatter_ctas),
                                             int(gather_ctas)))

    def buffers(self):
        """The batch's device buffers as CUDA torch tensors (views, no copy)."""
        import torch
        i = self.info()
        dev = torch.device("cuda", torch.cuda.current_device())

        def view(addr, n, dtype, shape):
            return _torch_view(addr, n, dtype, dev).view(*shape)

        n, s = self.n_total, len(self.counts)
        return {
            "xyzq": view(i.xyzq, 4 * n, torch.float32, (n, 4)),
            "energies": view(i.energies, s, torch.float64, (s,)),
            "forces": view(i.forces, 3 * n, torch.float64, (3, n)),
            "dLdE": view(i.dLdE, s, torch.float64, (s,)),
            "grad_forces": view(i.grad_forces, 3 * n, torch.float64, (3, n)),
            "grad_out": view(i.grad_out, 4 * n, torch.float64, (4, n)),
        }


def _torch_view(addr, numel, dtype, device):
    """A torch tensor over device memory the library owns (no copy, no ownership)."""
    import torch
    if numel == 0:
        return torch.empty(0, dtype=dtype, device=device)

    class _Iface:
        pass

    o = _Iface()
    typestr = {torch.float32: "<f4", torch.float64: "<f8"}[dtype]
    o.__cuda_array_interface__ = {"shape": (numel,), "typestr": typestr, "data": (addr, False),
                                  "version": 2, "strides": None}
    return torch.as_tensor(o, device=device)
