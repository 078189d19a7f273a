/*
 * gse_oracle.c -- CPU restatement of the GSE-k reciprocal-space path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
 * gse_b200/.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg load it; the product library never links or calls it.
 *
 * It restates, in plain C and in the same floating-point operation order, the
 * reference classes of ap-hynninen/GSE (paths relative to that project):
 *
 *   spreadChargeToGrid   CpuGaussCharge.cpp:235-384  (full (2n+1)^3 cube)
 *   interpolateLoop      CpuGaussCharge.cpp:105-172  (spherical cut r2 < rcut2)
 *   CpuGreensFuncGSE::mul CpuGreensFuncGSE.cpp:9-57
 *   CpuFFTSolver::run    CpuFFTSolver.cpp:75-96      (FFTW r2c -> mul -> c2r)
 *   CpuGSE::calculateEnergy CpuGSE.cpp:86-103
 *   CpuGSE::interpolateForce CpuGSE.cpp:70-80        (x ccelec afterwards)
 *   CpuGSE::setParam     CpuGSE.cpp:33-44
 *   spreadChargeOnGrid   CpuGaussCharge.cpp:390-519  (on-grid sigma convolution)
 *   calcElectricFieldOnGrid CpuGaussCharge.cpp:62-98
 *   calcDipoleSum        CpuGaussCharge.cpp:188-226
 *   CpuGSEk::spreadCharge1/solvePoisson/calculateEnergy CpuGSEk.cpp:30-58
 *   CpuEwaldRecip::calcForceEnergy CpuEwaldRecip.cpp:87-147
 *   CpuEwaldDirect::calcForceEnergy CpuEwaldDirect.cpp:45-131
 *
 * The reference links FFTW3 (double, FFTW_ESTIMATE) for the 3-D transforms;
 * FFTW is not vendored with the reference.  Its published transform
 * definitions are restated here with a project-written mixed-radix FFT:
 *   r2c:  X[kz][ky][kx] = sum_{z,y,x} x[z][y][x] exp(-2 pi i (kx x/nx + ky y/ny + kz z/nz)),
 *         kx = 0..nx/2 (the non-redundant half along the last, fastest axis);
 *   c2r:  the unnormalised inverse of the above under Hermitian symmetry,
 *         computed as complex inverse transforms along z and y followed by a
 *         per-row half-complex to real transform along x (imaginary parts of
 *         the self-conjugate x-bins are ignored, as FFTW's c2r does).
 * The transforms are pinned against numpy.fft (pocketfft) by the tests.
 *
 * Calculation type float: the reference calls unqualified exp()/round() on
 * float arguments, which resolve to the double overloads of <math.h>; the
 * Gaussian factors of its <double,float> instance are therefore evaluated in
 * double and rounded to float where they are stored (CpuGaussCharge.cpp:160,
 * :320-328, CpuGreensFuncGSE.cpp:50).  The float variants below use the same
 * double exp() with C's identical promotion rules.
 *
 * Where the reference is undefined (a stencil start more than one box length
 * below zero makes its `(i + size) % size` negative and indexes out of
 * bounds, CpuGaussCharge.cpp:364-366 and :148/:152/:156), this restatement
 * wraps periodically instead; inside the reference's defined domain the
 * result is the same.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846

static inline int pmod(int a, int m) {
  int r = a % m;
  return (r < 0) ? r + m : r;
}

/* ------------------------------------------------------------------------ */
/* Gaussian charge spreading, CpuGaussCharge.cpp:235-384                     */
/* ------------------------------------------------------------------------ */
#define DEFINE_SPREAD(SFX, CT, EXPFN)                                                  \
  int orc_spread_##SFX(int sizeX, int sizeY, int sizeZ, double sigma, double rcut,     \
                       int numCoord, const CT* xyzq, double boxx, double boxy,         \
                       double boxz, int normalize, CT* rho) {                          \
    const double hxd = boxx / (double)sizeX;                                           \
    const double hyd = boxy / (double)sizeY;                                           \
    const double hzd = boxz / (double)sizeZ;                                           \
    const int nx = (int)ceil(rcut / hxd);                                              \
    const int ny = (int)ceil(rcut / hyd);                                              \
    const int nz = (int)ceil(rcut / hzd);                                              \
    const CT inv_hx = (CT)(1.0 / hxd);                                                 \
    const CT inv_hy = (CT)(1.0 / hyd);                                                 \
    const CT inv_hz = (CT)(1.0 / hzd);                                                 \
    const CT hx = (CT)hxd;                                                             \
    const CT hy = (CT)hyd;                                                             \
    const CT hz = (CT)hzd;                                                             \
    const CT inv_2sigmasq = (CT)(1.0 / (2.0 * sigma * sigma));                         \
    const CT pref = (CT)pow(2.0 * ORC_PI * sigma * sigma, -3.0 / 2.0);                 \
    const long size = (long)sizeX * sizeY * sizeZ;                                     \
    for (long i = 0; i < size; i++) rho[i] = (CT)0;                                    \
    CT* wx = (CT*)malloc(sizeof(CT) * (2 * nx + 1));                                   \
    CT* wy = (CT*)malloc(sizeof(CT) * (2 * ny + 1));                                   \
    CT* wz = (CT*)malloc(sizeof(CT) * (2 * nz + 1));                                   \
    if (!wx || !wy || !wz) { free(wx); free(wy); free(wz); return -1; }                \
    for (int i = 0; i < numCoord; i++) {                                               \
      const CT x = xyzq[4 * i + 0];                                                    \
      const CT y = xyzq[4 * i + 1];                                                    \
      const CT z = xyzq[4 * i + 2];                                                    \
      const CT q_pref = xyzq[4 * i + 3] * pref;                                        \
      int ixc = (int)round(x * inv_hx) - nx;                                           \
      int iyc = (int)round(y * inv_hy) - ny;                                           \
      int izc = (int)round(z * inv_hz) - nz;                                           \
      const CT dx = ixc * hx - x;                                                      \
      const CT dy = iyc * hy - y;                                                      \
      const CT dz = izc * hz - z;                                                      \
      for (int j = 0; j <= 2 * nx; j++) { CT t = dx + j * hx; wx[j] = EXPFN(-t * t * inv_2sigmasq); } \
      for (int j = 0; j <= 2 * ny; j++) { CT t = dy + j * hy; wy[j] = EXPFN(-t * t * inv_2sigmasq); } \
      for (int j = 0; j <= 2 * nz; j++) { CT t = dz + j * hz; wz[j] = EXPFN(-t * t * inv_2sigmasq); } \
      if (normalize) {                                                                 \
        const CT pref1 = (CT)sqrt(2.0 * ORC_PI * sigma * sigma);                       \
        CT nrm = (CT)0;                                                                \
        for (int j = 0; j <= 2 * nx; j++) nrm += wx[j];                                \
        nrm = pref1 / nrm;                                                             \
        for (int j = 0; j <= 2 * nx; j++) wx[j] *= nrm;                                \
        nrm = (CT)0;                                                                   \
        for (int j = 0; j <= 2 * ny; j++) nrm += wy[j];                                \
        nrm = pref1 / nrm;                                                             \
        for (int j = 0; j <= 2 * ny; j++) wy[j] *= nrm;                                \
        nrm = (CT)0;                                                                   \
        for (int j = 0; j <= 2 * nz; j++) nrm += wz[j];                                \
        nrm = pref1 / nrm;                                                             \
        for (int j = 0; j <= 2 * nz; j++) wz[j] *= nrm;                                \
      }                                                                                \
      ixc = pmod(ixc, sizeX);                                                          \
      iyc = pmod(iyc, sizeY);                                                          \
      izc = pmod(izc, sizeZ);                                                          \
      for (int tz = 0; tz <= 2 * nz; tz++) {                                           \
        for (int ty = 0; ty <= 2 * ny; ty++) {                                         \
          for (int tx = 0; tx <= 2 * nx; tx++) {                                       \
            const int ix = (ixc + tx) % sizeX;                                         \
            const int iy = (iyc + ty) % sizeY;                                         \
            const int iz = (izc + tz) % sizeZ;                                         \
            const long p = ix + ((long)iy + (long)iz * sizeY) * sizeX;                 \
            rho[p] += q_pref * wx[tx] * wy[ty] * wz[tz];                               \
          }                                                                            \
        }                                                                              \
      }                                                                                \
    }                                                                                  \
    free(wx); free(wy); free(wz);                                                      \
    return 0;                                                                          \
  }

DEFINE_SPREAD(d, double, exp)
DEFINE_SPREAD(f, float, exp)

/* ------------------------------------------------------------------------ */
/* Gaussian gather (force interpolation), CpuGaussCharge.cpp:105-172         */
/* AT = double accumulation; CT = calculation type.                          */
/* ------------------------------------------------------------------------ */
#define DEFINE_GATHER(SFX, CT, EXPFN)                                                  \
  int orc_gather_##SFX(int sizeX, int sizeY, int sizeZ, double sigma, double rcut,     \
                       int numCoord, const CT* xyzq, double boxx, double boxy,         \
                       double boxz, const CT* phiData, double* resX, double* resY,     \
                       double* resZ) {                                                 \
    const double hxd = boxx / (double)sizeX;                                           \
    const double hyd = boxy / (double)sizeY;                                           \
    const double hzd = boxz / (double)sizeZ;                                           \
    const int nx = (int)ceil(rcut / hxd);                                              \
    const int ny = (int)ceil(rcut / hyd);                                              \
    const int nz = (int)ceil(rcut / hzd);                                              \
    const CT inv_hx = (CT)(1.0 / hxd);                                                 \
    const CT inv_hy = (CT)(1.0 / hyd);                                                 \
    const CT inv_hz = (CT)(1.0 / hzd);                                                 \
    const CT hx = (CT)hxd;                                                             \
    const CT hy = (CT)hyd;                                                             \
    const CT hz = (CT)hzd;                                                             \
    const CT rcut2 = (CT)(rcut * rcut);                                                \
    const CT inv_2sigmasq = (CT)(1.0 / (2.0 * sigma * sigma));                         \
    const CT pref = (CT)(pow(2.0 * ORC_PI, -3.0 / 2.0) * hxd * hyd * hzd * pow(sigma, -5.0)); \
    _Pragma("omp parallel for schedule(static)")                                       \
    for (int i = 0; i < numCoord; i++) {                                               \
      const CT x = xyzq[4 * i + 0];                                                    \
      const CT y = xyzq[4 * i + 1];                                                    \
      const CT z = xyzq[4 * i + 2];                                                    \
      const CT fac = xyzq[4 * i + 3] * pref;                                           \
      const int ix = (int)round(x * inv_hx);                                           \
      const int iy = (int)round(y * inv_hy);                                           \
      const int iz = (int)round(z * inv_hz);                                           \
      double rx = 0.0, ry = 0.0, rz = 0.0;                                             \
      for (int tz = iz - nz; tz <= iz + nz; tz++) {                                    \
        const CT zp = ((CT)tz) * hz;                                                   \
        const CT dz = z - zp;                                                          \
        const int pz = pmod(tz, sizeZ);                                                \
        for (int ty = iy - ny; ty <= iy + ny; ty++) {                                  \
          const CT yp = ((CT)ty) * hy;                                                 \
          const CT dy = y - yp;                                                        \
          const int py = pmod(ty, sizeY);                                              \
          for (int tx = ix - nx; tx <= ix + nx; tx++) {                                \
            const CT xp = ((CT)tx) * hx;                                               \
            const CT dx = x - xp;                                                      \
            const int px = pmod(tx, sizeX);                                            \
            const CT r2 = dx * dx + dy * dy + dz * dz;                                 \
            if (r2 < rcut2) {                                                          \
              const long p = px + ((long)py + (long)pz * sizeY) * sizeX;               \
              const CT r = fac * EXPFN(-r2 * inv_2sigmasq) * phiData[p];               \
              rx += (double)(r * dx);                                                  \
              ry += (double)(r * dy);                                                  \
              rz += (double)(r * dz);                                                  \
            }                                                                          \
          }                                                                            \
        }                                                                              \
      }                                                                                \
      resX[i] = rx;                                                                    \
      resY[i] = ry;                                                                    \
      resZ[i] = rz;                                                                    \
    }                                                                                  \
    return 0;                                                                          \
  }

DEFINE_GATHER(d, double, exp)
DEFINE_GATHER(f, float, exp)

/* ------------------------------------------------------------------------ */
/* k-space Green's function multiply, CpuGreensFuncGSE.cpp:9-57              */
/* rho: interleaved complex half spectrum [nfftZ][nfftY][nfftX/2+1].         */
/* ------------------------------------------------------------------------ */
#define DEFINE_GREEN(SFX, T, EXPFN)                                                    \
  void orc_green_mul_##SFX(int nfftX, int nfftY, int nfftZ, double boxx, double boxy,  \
                           double boxz, double sigma, T* rhoData) {                    \
    const int sizeX = nfftX / 2 + 1;                                                   \
    const int sizeY = nfftY;                                                           \
    const int sizeZ = nfftZ;                                                           \
    const int halfNfftX = nfftX / 2 + (nfftX % 2);                                     \
    const int halfNfftY = nfftY / 2 + (nfftY % 2);                                     \
    const int halfNfftZ = nfftZ / 2 + (nfftZ % 2);                                     \
    const T twopi_boxx = (T)(2.0 * ORC_PI / boxx);                                     \
    const T twopi_boxy = (T)(2.0 * ORC_PI / boxy);                                     \
    const T twopi_boxz = (T)(2.0 * ORC_PI / boxz);                                     \
    const T fourpi_vol = (T)(4.0 * ORC_PI / (double)(nfftX * nfftY * nfftZ));          \
    const T sigmafac = (T)(sigma * sigma / 2.0);                                       \
    long p = 0;                                                                        \
    for (int iz = 0; iz < sizeZ; iz++) {                                               \
      for (int iy = 0; iy < sizeY; iy++) {                                             \
        for (int ix = 0; ix < sizeX; ix++, p += 2) {                                   \
          if (p == 0) { rhoData[0] = (T)0; rhoData[1] = (T)0; continue; }              \
          const int kx = (ix >= halfNfftX) ? ix - nfftX : ix;                          \
          const int ky = (iy >= halfNfftY) ? iy - nfftY : iy;                          \
          const int kz = (iz >= halfNfftZ) ? iz - nfftZ : iz;                          \
          const T kxd = ((T)kx) * twopi_boxx;                                          \
          const T kyd = ((T)ky) * twopi_boxy;                                          \
          const T kzd = ((T)kz) * twopi_boxz;                                          \
          const T kd2 = kxd * kxd + kyd * kyd + kzd * kzd;                             \
          const T fac = fourpi_vol * EXPFN(-sigmafac * kd2) / kd2;                     \
          rhoData[p] *= fac;                                                           \
          rhoData[p + 1] *= fac;                                                       \
        }                                                                              \
      }                                                                                \
    }                                                                                  \
  }

DEFINE_GREEN(d, double, exp)
DEFINE_GREEN(f, float, exp)

/* ------------------------------------------------------------------------ */
/* Mesh energy, CpuGSE.cpp:86-103 (AT = double)                              */
/* ------------------------------------------------------------------------ */
#define DEFINE_ENERGY(SFX, CT)                                                         \
  double orc_energy_##SFX(int sizeX, int sizeY, int sizeZ, double boxx, double boxy,   \
                          double boxz, double ccelec, const CT* rho, const CT* phi) {  \
    const long size = (long)sizeX * sizeY * sizeZ;                                     \
    double energy = 0.0;                                                               \
    for (long i = 0; i < size; i++) energy += (double)(rho[i] * phi[i]);               \
    const double hx = boxx / (double)sizeX;                                            \
    const double hy = boxy / (double)sizeY;                                            \
    const double hz = boxz / (double)sizeZ;                                            \
    energy *= ccelec * hx * hy * hz * 0.5;                                             \
    return energy;                                                                     \
  }

DEFINE_ENERGY(d, double)
DEFINE_ENERGY(f, float)

/* ------------------------------------------------------------------------ */
/* On-grid Gaussian convolution, CpuGaussCharge.cpp:390-519.  Three periodic */
/* 1-D passes, x then y then z, with taps G[i] = exp(-h^2 i^2 / (2 sigma^2)),*/
/* i = -n..n, n = ceil(rcut / h) per axis; the z taps also carry             */
/* (2 pi sigma^2)^(-3/2) hx hy hz (the product formed in double, as the      */
/* reference's float * double(exp) does).  Every output is summed from zero  */
/* in tap order, each product and sum rounded in CT.                         */
/* ------------------------------------------------------------------------ */
#define DEFINE_CONV(SFX, CT, EXPFN)                                                    \
  int orc_spread_on_grid_##SFX(int sizeX, int sizeY, int sizeZ, double sigma,          \
                               double rcut, double boxx, double boxy, double boxz,     \
                               const CT* rho, CT* rhoS) {                              \
    const double hxd = boxx / (double)sizeX;                                           \
    const double hyd = boxy / (double)sizeY;                                           \
    const double hzd = boxz / (double)sizeZ;                                           \
    const int nx = (int)ceil(rcut / hxd);                                              \
    const int ny = (int)ceil(rcut / hyd);                                              \
    const int nz = (int)ceil(rcut / hzd);                                              \
    const CT inv_2sigmasq = (CT)(1.0 / (2.0 * sigma * sigma));                         \
    const CT pref = (CT)(pow(2.0 * ORC_PI * sigma * sigma, -3.0 / 2.0) * hxd * hyd * hzd); \
    const CT hxsq = (CT)(hxd * hxd);                                                   \
    const CT hysq = (CT)(hyd * hyd);                                                   \
    const CT hzsq = (CT)(hzd * hzd);                                                   \
    const long size = (long)sizeX * sizeY * sizeZ;                                     \
    CT* gx = (CT*)malloc(sizeof(CT) * (2 * nx + 1));                                   \
    CT* gy = (CT*)malloc(sizeof(CT) * (2 * ny + 1));                                   \
    CT* gz = (CT*)malloc(sizeof(CT) * (2 * nz + 1));                                   \
    CT* tx = (CT*)malloc(sizeof(CT) * size);                                           \
    CT* txy = (CT*)malloc(sizeof(CT) * size);                                          \
    if (!gx || !gy || !gz || !tx || !txy) {                                            \
      free(gx); free(gy); free(gz); free(tx); free(txy);                               \
      return -1;                                                                       \
    }                                                                                  \
    for (int i = -nx; i <= nx; i++) gx[i + nx] = EXPFN(-hxsq * (CT)(i * i) * inv_2sigmasq); \
    for (int i = -ny; i <= ny; i++) gy[i + ny] = EXPFN(-hysq * (CT)(i * i) * inv_2sigmasq); \
    for (int i = -nz; i <= nz; i++)                                                    \
      gz[i + nz] = pref * EXPFN(-hzsq * (CT)(i * i) * inv_2sigmasq);                   \
    for (int z = 0; z < sizeZ; z++)                                                    \
      for (int y = 0; y < sizeY; y++) {                                                \
        const long row = ((long)y + (long)z * sizeY) * sizeX;                          \
        for (int x = 0; x < sizeX; x++) {                                              \
          CT s = (CT)0;                                                                \
          for (int i = -nx; i <= nx; i++) s += gx[i + nx] * rho[row + pmod(x + i, sizeX)]; \
          tx[row + x] = s;                                                             \
        }                                                                              \
      }                                                                                \
    for (int z = 0; z < sizeZ; z++)                                                    \
      for (int x = 0; x < sizeX; x++)                                                  \
        for (int y = 0; y < sizeY; y++) {                                              \
          CT s = (CT)0;                                                                \
          for (int i = -ny; i <= ny; i++)                                              \
            s += gy[i + ny] * tx[x + ((long)pmod(y + i, sizeY) + (long)z * sizeY) * sizeX]; \
          txy[x + ((long)y + (long)z * sizeY) * sizeX] = s;                            \
        }                                                                              \
    for (int x = 0; x < sizeX; x++)                                                    \
      for (int y = 0; y < sizeY; y++)                                                  \
        for (int z = 0; z < sizeZ; z++) {                                              \
          CT s = (CT)0;                                                                \
          for (int i = -nz; i <= nz; i++)                                              \
            s += gz[i + nz] * txy[x + ((long)y + (long)pmod(z + i, sizeZ) * sizeY) * sizeX]; \
          rhoS[x + ((long)y + (long)z * sizeY) * sizeX] = s;                           \
        }                                                                              \
    free(gx); free(gy); free(gz); free(tx); free(txy);                                 \
    return 0;                                                                          \
  }

DEFINE_CONV(d, double, exp)
DEFINE_CONV(f, float, exp)

/* ------------------------------------------------------------------------ */
/* Electric field on the grid, CpuGaussCharge.cpp:62-98: forward differences */
/* E = -(phi(p + e_d) - phi(p)) / h_d, periodic, in CT.                      */
/* ------------------------------------------------------------------------ */
#define DEFINE_EFIELD(SFX, CT)                                                         \
  void orc_efield_##SFX(int sizeX, int sizeY, int sizeZ, double boxx, double boxy,     \
                        double boxz, const CT* phi, CT* Ex, CT* Ey, CT* Ez) {          \
    const CT inv_hx = (CT)(1.0 / (boxx / (double)sizeX));                              \
    const CT inv_hy = (CT)(1.0 / (boxy / (double)sizeY));                              \
    const CT inv_hz = (CT)(1.0 / (boxz / (double)sizeZ));                              \
    for (int z = 0; z < sizeZ; z++)                                                    \
      for (int y = 0; y < sizeY; y++)                                                  \
        for (int x = 0; x < sizeX; x++) {                                              \
          const long p = x + ((long)y + (long)z * sizeY) * sizeX;                      \
          const CT c = phi[p];                                                         \
          const CT px = phi[pmod(x + 1, sizeX) + ((long)y + (long)z * sizeY) * sizeX]; \
          const CT py = phi[x + ((long)pmod(y + 1, sizeY) + (long)z * sizeY) * sizeX]; \
          const CT pz = phi[x + ((long)y + (long)pmod(z + 1, sizeZ) * sizeY) * sizeX]; \
          Ex[p] = -(px - c) * inv_hx;                                                  \
          Ey[p] = -(py - c) * inv_hy;                                                  \
          Ez[p] = -(pz - c) * inv_hz;                                                  \
        }                                                                              \
  }

DEFINE_EFIELD(d, double)
DEFINE_EFIELD(f, float)

/* ------------------------------------------------------------------------ */
/* Dipole sum of a charge grid, CpuGaussCharge.cpp:188-226: sum over points  */
/* of (rho hx hy hz) * (hx ix, hy iy, hz iz), each term formed in CT and     */
/* added in double in z, y, x loop order.                                    */
/* ------------------------------------------------------------------------ */
#define DEFINE_DIPOLE(SFX, CT)                                                         \
  void orc_dipole_##SFX(int sizeX, int sizeY, int sizeZ, double boxx, double boxy,     \
                        double boxz, const CT* rho, double* dip) {                     \
    const CT hx = (CT)(boxx / (double)sizeX);                                          \
    const CT hy = (CT)(boxy / (double)sizeY);                                          \
    const CT hz = (CT)(boxz / (double)sizeZ);                                          \
    double sx = 0.0, sy = 0.0, sz = 0.0;                                               \
    for (int iz = 0; iz < sizeZ; iz++) {                                               \
      const CT z = hz * (CT)iz;                                                        \
      for (int iy = 0; iy < sizeY; iy++) {                                             \
        const CT y = hy * (CT)iy;                                                      \
        for (int ix = 0; ix < sizeX; ix++) {                                           \
          const CT x = hx * (CT)ix;                                                    \
          const CT val = rho[ix + ((long)iy + (long)iz * sizeY) * sizeX] * hx * hy * hz; \
          sx += (double)(val * x);                                                     \
          sy += (double)(val * y);                                                     \
          sz += (double)(val * z);                                                     \
        }                                                                              \
      }                                                                                \
    }                                                                                  \
    dip[0] = sx;                                                                       \
    dip[1] = sy;                                                                       \
    dip[2] = sz;                                                                       \
  }

DEFINE_DIPOLE(d, double)
DEFINE_DIPOLE(f, float)

/* ------------------------------------------------------------------------ */
/* Project-written complex FFT (recursive mixed radix, any length).          */
/* ------------------------------------------------------------------------ */
typedef struct { double re, im; } ocpx;

typedef struct {
  int n;
  int nf;
  int f[40];
  ocpx* w; /* w[j] = exp(-2 pi i j / n) */
} fft1_plan;

static int fft1_plan_init(fft1_plan* p, int n) {
  p->n = n;
  p->nf = 0;
  int m = n;
  for (int d = 2; m > 1;) {
    if (m % d == 0) { p->f[p->nf++] = d; m /= d; } else { d = (d == 2) ? 3 : d + 2; }
  }
  p->w = (ocpx*)malloc(sizeof(ocpx) * (n > 0 ? n : 1));
  if (!p->w) return -1;
  for (int j = 0; j < n; j++) {
    const double a = -2.0 * ORC_PI * (double)j / (double)n;
    p->w[j].re = cos(a);
    p->w[j].im = sin(a);
  }
  return 0;
}

static void fft1_plan_free(fft1_plan* p) { free(p->w); p->w = NULL; }

/* W_n^e for the plan of length N, sign -1 forward / +1 inverse */
static inline ocpx twid(const fft1_plan* P, long e, int n, int inverse) {
  const long idx = (e % n) * (long)(P->n / n);
  ocpx w = P->w[idx];
  if (inverse) w.im = -w.im;
  return w;
}

/* y[0..n-1] = DFT_n(x[0], x[xs], ..., x[(n-1) xs]) */
static void fft1_rec(const fft1_plan* P, const ocpx* x, long xs, ocpx* y, int n, int lev,
                     int inverse, ocpx* t) {
  if (n == 1) { y[0] = x[0]; return; }
  const int p = P->f[lev];
  const int m = n / p;
  for (int r = 0; r < p; r++) fft1_rec(P, x + r * xs, xs * p, y + (long)r * m, m, lev + 1, inverse, t);
  for (int k = 0; k < m; k++) {
    for (int r = 0; r < p; r++) {
      const ocpx a = y[(long)r * m + k];
      const ocpx w = twid(P, (long)r * k, n, inverse);
      t[r].re = a.re * w.re - a.im * w.im;
      t[r].im = a.re * w.im + a.im * w.re;
    }
    for (int q = 0; q < p; q++) {
      double sr = 0.0, si = 0.0;
      for (int r = 0; r < p; r++) {
        const ocpx w = twid(P, (long)r * q * m, n, inverse);
        sr += t[r].re * w.re - t[r].im * w.im;
        si += t[r].re * w.im + t[r].im * w.re;
      }
      y[k + (long)q * m].re = sr;
      y[k + (long)q * m].im = si;
    }
  }
}

static int max_factor(const fft1_plan* p) {
  int mx = 1;
  for (int i = 0; i < p->nf; i++) if (p->f[i] > mx) mx = p->f[i];
  return mx;
}

/* Length-n complex DFT of a strided vector, in place through a buffer. */
static void fft1_strided(const fft1_plan* P, ocpx* data, long stride, int inverse, ocpx* in,
                         ocpx* out, ocpx* t) {
  const int n = P->n;
  for (int j = 0; j < n; j++) in[j] = data[j * stride];
  fft1_rec(P, in, 1, out, n, 0, inverse, t);
  for (int j = 0; j < n; j++) data[j * stride] = out[j];
}

/* 3-D r2c with FFTW's conventions: in real [nz][ny][nx], out complex
 * [nz][ny][nx/2+1] interleaved (re, im). */
int orc_fft_r2c_3d(int nx, int ny, int nz, const double* in, double* outd) {
  const int nxh = nx / 2 + 1;
  ocpx* out = (ocpx*)outd;
  fft1_plan px, py, pz;
  if (fft1_plan_init(&px, nx) || fft1_plan_init(&py, ny) || fft1_plan_init(&pz, nz)) return -1;
  const int nmax = (nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz));
  const int fmax = max_factor(&px) > max_factor(&py) ? max_factor(&px) : max_factor(&py);
  const int fm = fmax > max_factor(&pz) ? fmax : max_factor(&pz);
#pragma omp parallel
  {
    ocpx* a = (ocpx*)malloc(sizeof(ocpx) * nmax);
    ocpx* b = (ocpx*)malloc(sizeof(ocpx) * nmax);
    ocpx* t = (ocpx*)malloc(sizeof(ocpx) * fm);
#pragma omp for schedule(static)
    for (long row = 0; row < (long)ny * nz; row++) {
      const double* r = in + row * nx;
      for (int j = 0; j < nx; j++) { a[j].re = r[j]; a[j].im = 0.0; }
      fft1_rec(&px, a, 1, b, nx, 0, 0, t);
      memcpy(out + row * nxh, b, sizeof(ocpx) * nxh);
    }
#pragma omp for schedule(static)
    for (long c = 0; c < (long)nz * nxh; c++) {
      const long z = c / nxh, kx = c % nxh;
      fft1_strided(&py, out + z * (long)ny * nxh + kx, nxh, 0, a, b, t);
    }
#pragma omp for schedule(static)
    for (long c = 0; c < (long)ny * nxh; c++) {
      fft1_strided(&pz, out + c, (long)ny * nxh, 0, a, b, t);
    }
    free(a); free(b); free(t);
  }
  fft1_plan_free(&px); fft1_plan_free(&py); fft1_plan_free(&pz);
  return 0;
}

/* 3-D c2r (unnormalised inverse of the above).  `ind` is not modified. */
int orc_fft_c2r_3d(int nx, int ny, int nz, const double* ind, double* out) {
  const int nxh = nx / 2 + 1;
  const long nc = (long)nxh * ny * nz;
  ocpx* w = (ocpx*)malloc(sizeof(ocpx) * nc);
  if (!w) return -1;
  memcpy(w, ind, sizeof(ocpx) * nc);
  fft1_plan px, py, pz;
  if (fft1_plan_init(&px, nx) || fft1_plan_init(&py, ny) || fft1_plan_init(&pz, nz)) { free(w); return -1; }
  const int nmax = (nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz));
  const int fmax = max_factor(&px) > max_factor(&py) ? max_factor(&px) : max_factor(&py);
  const int fm = fmax > max_factor(&pz) ? fmax : max_factor(&pz);
#pragma omp parallel
  {
    ocpx* a = (ocpx*)malloc(sizeof(ocpx) * nmax);
    ocpx* b = (ocpx*)malloc(sizeof(ocpx) * nmax);
    ocpx* t = (ocpx*)malloc(sizeof(ocpx) * fm);
#pragma omp for schedule(static)
    for (long c = 0; c < (long)ny * nxh; c++) {
      fft1_strided(&pz, w + c, (long)ny * nxh, 1, a, b, t);
    }
#pragma omp for schedule(static)
    for (long c = 0; c < (long)nz * nxh; c++) {
      const long z = c / nxh, kx = c % nxh;
      fft1_strided(&py, w + z * (long)ny * nxh + kx, nxh, 1, a, b, t);
    }
#pragma omp for schedule(static)
    for (long row = 0; row < (long)ny * nz; row++) {
      const ocpx* h = w + row * nxh;
      for (int k = 0; k < nxh; k++) a[k] = h[k];
      for (int k = nxh; k < nx; k++) { a[k].re = h[nx - k].re; a[k].im = -h[nx - k].im; }
      fft1_rec(&px, a, 1, b, nx, 0, 1, t);
      double* r = out + row * nx;
      for (int j = 0; j < nx; j++) r[j] = b[j].re;
    }
    free(a); free(b); free(t);
  }
  fft1_plan_free(&px); fft1_plan_free(&py); fft1_plan_free(&pz);
  free(w);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Full GSE-k force evaluation <AT=double, CT=double>, as cpu_gse runs it:   */
/* spreadCharge1 -> solvePoisson -> calculateEnergy -> interpolateForce      */
/* (CpuGSEk.cpp:30-58, CpuGSE.cpp:33-44,70-103).                             */
/* rhoS_out / phi_out / rhoK_out may be NULL.                                */
/* ------------------------------------------------------------------------ */
int orc_gsek_forward_d(int sx, int sy, int sz, double sigma, double kappa, double lambdaSigma1,
                       double boxx, double boxy, double boxz, double ccelec, int n,
                       const double* xyzq, double* energy, double* fx, double* fy, double* fz,
                       double* rhoS_out, double* phi_out) {
  if (kappa < 0.0 || kappa > 0.5) return -2;
  const double sigma1 = sigma * sqrt(kappa);
  const double sigma2 = sigma * sqrt(1.0 - 2.0 * kappa);
  const double rcut1 = lambdaSigma1 * sqrt(2.0) * sigma1;
  const long size = (long)sx * sy * sz;
  const long ksize = (long)(sx / 2 + 1) * 2 * sy * sz;
  double* rhoS = (double*)malloc(sizeof(double) * size);
  double* phi = (double*)malloc(sizeof(double) * size);
  double* rhoK = (double*)malloc(sizeof(double) * ksize);
  int rc = -1;
  if (!rhoS || !phi || !rhoK) goto done;
  if (orc_spread_d(sx, sy, sz, sigma1, rcut1, n, xyzq, boxx, boxy, boxz, 0, rhoS)) goto done;
  if (orc_fft_r2c_3d(sx, sy, sz, rhoS, rhoK)) goto done;
  orc_green_mul_d(sx, sy, sz, boxx, boxy, boxz, sigma2, rhoK);
  if (orc_fft_c2r_3d(sx, sy, sz, rhoK, phi)) goto done;
  *energy = orc_energy_d(sx, sy, sz, boxx, boxy, boxz, ccelec, rhoS, phi);
  if (fx && fy && fz) {
    orc_gather_d(sx, sy, sz, sigma1, rcut1, n, xyzq, boxx, boxy, boxz, phi, fx, fy, fz);
    for (int i = 0; i < n; i++) {
      fx[i] *= ccelec;
      fy[i] *= ccelec;
      fz[i] *= ccelec;
    }
  }
  if (rhoS_out) memcpy(rhoS_out, rhoS, sizeof(double) * size);
  if (phi_out) memcpy(phi_out, phi, sizeof(double) * size);
  rc = 0;
done:
  free(rhoS); free(phi); free(rhoK);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Ewald reciprocal sum, CpuEwaldRecip.cpp:87-147.                           */
/* E = sum_{k != 0, |k|_int <= kcut} (2 pi / V) ccelec exp(-sigma^2 k^2/2)/k^2 |S(k)|^2
 * with S(k) = sum_i q_i exp(i k.r_i); F_i = -dE/dr_i.                       */
/* The same sum is evaluated over the half space of k (k and -k contribute  */
/* equally) with the phase factors exp(i kx x) built by complex recurrence   */
/* along kx: the mathematics of the reference, with O(N K^3) complex        */
/* multiplies instead of O(N K^3) sin/cos calls.                             */
/* fx/fy/fz may be NULL (energy only).                                      */
/* ------------------------------------------------------------------------ */
double orc_ewald_recip(double sigma, int kcut, double boxx, double boxy, double boxz,
                       double ccelec, int n, const double* xyzq, double* fx, double* fy,
                       double* fz) {
  const double inv_boxx = 1.0 / boxx, inv_boxy = 1.0 / boxy, inv_boxz = 1.0 / boxz;
  const double half_sigmasq = 0.5 * sigma * sigma;
  const double pref = 2.0 * ORC_PI * inv_boxx * inv_boxy * inv_boxz * ccelec;
  const int kcut2 = kcut * kcut;
  const int do_force = (fx && fy && fz);
  /* rows of the half space: (kz, ky) with kz > 0, or kz == 0 and ky >= 0 */
  const int nrows_max = (kcut + 1) * (2 * kcut + 1);
  int* rkz = (int*)malloc(sizeof(int) * nrows_max);
  int* rky = (int*)malloc(sizeof(int) * nrows_max);
  int nrows = 0;
  for (int kz = 0; kz <= kcut; kz++)
    for (int ky = (kz == 0 ? 0 : -kcut); ky <= kcut; ky++)
      if (ky * ky + kz * kz <= kcut2) { rkz[nrows] = kz; rky[nrows] = ky; nrows++; }
  double E = 0.0;
  int nthr = 1;
#ifdef _OPENMP
  nthr = omp_get_max_threads();
#endif
  double* facc = NULL;
  if (do_force) facc = (double*)calloc((size_t)nthr * 3 * n, sizeof(double));
  ocpx* ux = (ocpx*)malloc(sizeof(ocpx) * n);
  for (int i = 0; i < n; i++) {
    const double a = 2.0 * ORC_PI * xyzq[4 * i] * inv_boxx;
    ux[i].re = cos(a);
    ux[i].im = sin(a);
  }
#pragma omp parallel reduction(+ : E)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* f = do_force ? facc + (size_t)tid * 3 * n : NULL;
    ocpx* S = (ocpx*)malloc(sizeof(ocpx) * (2 * kcut + 1));
    double* P = (double*)malloc(sizeof(double) * (2 * kcut + 1));
#pragma omp for schedule(dynamic, 1)
    for (int r = 0; r < nrows; r++) {
      const int kz = rkz[r], ky = rky[r];
      const int rem = kcut2 - ky * ky - kz * kz;
      int kxm = (int)floor(sqrt((double)rem));
      while (kxm * kxm > rem) kxm--;
      while ((kxm + 1) * (kxm + 1) <= rem) kxm++;
      const int kx0 = (kz == 0 && ky == 0) ? 1 : -kxm;
      const int nk = kxm - kx0 + 1;
      if (nk <= 0) continue;
      const double kzv = 2.0 * ORC_PI * (double)kz * inv_boxz;
      const double kyv = 2.0 * ORC_PI * (double)ky * inv_boxy;
      for (int j = 0; j < nk; j++) { S[j].re = 0.0; S[j].im = 0.0; }
      for (int i = 0; i < n; i++) {
        const double ph = kyv * xyzq[4 * i + 1] + kzv * xyzq[4 * i + 2] +
                          2.0 * ORC_PI * (double)kx0 * inv_boxx * xyzq[4 * i];
        const double q = xyzq[4 * i + 3];
        double er = q * cos(ph), ei = q * sin(ph);
        const double wr = ux[i].re, wi = ux[i].im;
        for (int j = 0; j < nk; j++) {
          S[j].re += er;
          S[j].im += ei;
          const double tr = er * wr - ei * wi;
          ei = er * wi + ei * wr;
          er = tr;
        }
      }
      for (int j = 0; j < nk; j++) {
        const int kx = kx0 + j;
        const double kxv = 2.0 * ORC_PI * (double)kx * inv_boxx;
        const double ksq = kxv * kxv + kyv * kyv + kzv * kzv;
        P[j] = pref * exp(-ksq * half_sigmasq) / ksq;
        E += 2.0 * P[j] * (S[j].re * S[j].re + S[j].im * S[j].im);
      }
      if (do_force) {
        for (int i = 0; i < n; i++) {
          const double ph = kyv * xyzq[4 * i + 1] + kzv * xyzq[4 * i + 2] +
                            2.0 * ORC_PI * (double)kx0 * inv_boxx * xyzq[4 * i];
          const double q = xyzq[4 * i + 3];
          double er = cos(ph), ei = sin(ph);
          const double wr = ux[i].re, wi = ux[i].im;
          double ax = 0.0, ayz = 0.0;
          for (int j = 0; j < nk; j++) {
            /* Im(conj(S) e^{i k.r}) = S_re sin - S_im cos */
            const double im = S[j].re * ei - S[j].im * er;
            const double t = P[j] * im;
            ax += t * 2.0 * ORC_PI * (double)(kx0 + j) * inv_boxx;
            ayz += t;
            const double tr = er * wr - ei * wi;
            ei = er * wi + ei * wr;
            er = tr;
          }
          /* F_i = sum_k 2 P q k Im(conj(S) e^{ik r}), doubled for -k */
          f[3 * i + 0] += 4.0 * q * ax;
          f[3 * i + 1] += 4.0 * q * ayz * kyv;
          f[3 * i + 2] += 4.0 * q * ayz * kzv;
        }
      }
    }
    free(S); free(P);
  }
  if (do_force) {
    for (int i = 0; i < n; i++) {
      double sx = 0.0, sy = 0.0, sz = 0.0;
      for (int t = 0; t < nthr; t++) {
        sx += facc[(size_t)t * 3 * n + 3 * i + 0];
        sy += facc[(size_t)t * 3 * n + 3 * i + 1];
        sz += facc[(size_t)t * 3 * n + 3 * i + 2];
      }
      fx[i] = sx;
      fy[i] = sy;
      fz[i] = sz;
    }
  }
  free(facc); free(ux); free(rkz); free(rky);
  return E;
}

/* ------------------------------------------------------------------------ */
/* Ewald direct sum with self energy, CpuEwaldDirect.cpp:45-131, with the   */
/* exclusion lists of setupExclusions (CpuEwaldDirect.cpp:31-40) when        */
/* n_iblo14 > 0: the pair (j, i), j < i, is skipped when i + 1 equals        */
/* |inb14[k]| for some k in [iblo14[j-1], iblo14[j]) (:71-85).               */
/* ------------------------------------------------------------------------ */
double orc_ewald_direct(double sigma, double rcut, double boxx, double boxy, double boxz,
                        double ccelec, int n, const double* xyzq, int n_iblo14,
                        const int* iblo14, const int* inb14, double* fx, double* fy,
                        double* fz) {
  const double rcut2 = rcut * rcut;
  const double hboxx = 0.5 * boxx, hboxy = 0.5 * boxy, hboxz = 0.5 * boxz;
  const double inv_sqrt2sigma = 1.0 / (sqrt(2.0) * sigma);
  const double inv_2sigmasq = 1.0 / (2.0 * sigma * sigma);
  const double two_sqrtpi = 2.0 / sqrt(ORC_PI);
  for (int i = 0; i < n; i++) { fx[i] = 0.0; fy[i] = 0.0; fz[i] = 0.0; }
  double E = 0.0;
  for (int j = 0; j < n - 1; j++) {
    const double xj = xyzq[4 * j], yj = xyzq[4 * j + 1], zj = xyzq[4 * j + 2];
    const double qj = xyzq[4 * j + 3] * ccelec;
    const int ex0 = (n_iblo14 > 0 && j >= 1) ? iblo14[j - 1] : 0;
    const int ex1 = n_iblo14 > 0 ? iblo14[j] : 0;
    for (int i = j + 1; i < n; i++) {
      int skip = 0;
      for (int k = ex0; k < ex1 && !skip; k++) skip = (abs(inb14[k]) - 1 == i);
      if (skip) continue;
      double dx = xyzq[4 * i] - xj, dy = xyzq[4 * i + 1] - yj, dz = xyzq[4 * i + 2] - zj;
      while (dx < -hboxx) dx += boxx;
      while (dx > hboxx) dx -= boxx;
      while (dy < -hboxy) dy += boxy;
      while (dy > hboxy) dy -= boxy;
      while (dz < -hboxz) dz += boxz;
      while (dz > hboxz) dz -= boxz;
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < rcut2) {
        const double qq = qj * xyzq[4 * i + 3];
        const double r = sqrt(r2);
        const double erfcval = erfc(r * inv_sqrt2sigma);
        const double expval = exp(-r2 * inv_2sigmasq);
        const double f = -qq * (two_sqrtpi * inv_sqrt2sigma * expval + erfcval / r) / r2;
        fx[i] += f * dx; fy[i] += f * dy; fz[i] += f * dz;
        fx[j] -= f * dx; fy[j] -= f * dy; fz[j] -= f * dz;
        E += qq * erfcval / r;
      }
    }
  }
  double Eself = 0.0;
  for (int i = 0; i < n; i++) Eself += xyzq[4 * i + 3] * xyzq[4 * i + 3];
  Eself *= -ccelec / sqrt(2.0 * ORC_PI * sigma * sigma);
  return E + Eself;
}
