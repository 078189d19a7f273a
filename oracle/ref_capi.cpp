// ref_capi.cpp -- extern "C" wrapper around the reference's own CPU classes
// (ap-hynninen/GSE: CpuGSEk, CpuGaussCharge, CpuGreensFuncGSE, CpuEwaldRecip,
// CpuEwaldDirect), compiled unchanged from the reference sources by
// oracle/Makefile into oracle/_ref/libgse_ref.so.
//
// Test infrastructure: tests/ use it to pin the C restatement in
// gse_oracle.c, and bench.py times it as the reference CPU baseline.  The
// product library never links it.
#include <cstring>
#include <fstream>
#include <iostream>

#include "CpuEwaldDirect.h"
#include "CpuEwaldRecip.h"
#include "CpuGSEk.h"
#include "CpuGaussCharge.h"
#include "CpuGreensFuncGSE.h"

extern "C" {

// One full force evaluation exactly as cpu_gse's testRandom/test48K run it
// (cpu_gse.cpp:440-455): spreadCharge1 -> solvePoisson -> calculateEnergy ->
// interpolateForce on CpuGSEk<double,double>.
int ref_gsek_forward_dd(int sx, int sy, int sz, double sigma, double kappa, double lambdaSigma,
                        double lambdaSigma1, double boxx, double boxy, double boxz,
                        double ccelec, int n, const double* xyzq, double* energy, double* fx,
                        double* fy, double* fz, double* rhoS_out, double* phi_out) {
  CpuGSEk<double, double> g(sx, sy, sz, sigma, kappa, lambdaSigma, lambdaSigma1, boxx, boxy,
                            boxz, ccelec);
  const xyzq_t<double>* p = reinterpret_cast<const xyzq_t<double>*>(xyzq);
  g.spreadCharge1(n, p);
  g.solvePoisson();
  *energy = g.calculateEnergy();
  g.interpolateForce(n, p, fx, fy, fz);
  const size_t size = (size_t)sx * sy * sz;
  if (rhoS_out) std::memcpy(rhoS_out, g.getRhoS().getDataPointer(), size * sizeof(double));
  if (phi_out) std::memcpy(phi_out, g.getPhi().getDataPointer(), size * sizeof(double));
  return 0;
}

// Persistent object for repeated evaluations (the CPU baseline timing loop).
void* ref_gsek_create(int sx, int sy, int sz, double sigma, double kappa, double lambdaSigma,
                      double lambdaSigma1, double boxx, double boxy, double boxz,
                      double ccelec) {
  return new CpuGSEk<double, double>(sx, sy, sz, sigma, kappa, lambdaSigma, lambdaSigma1, boxx,
                                     boxy, boxz, ccelec);
}

int ref_gsek_eval(void* h, int n, const double* xyzq, double* energy, double* fx, double* fy,
                  double* fz) {
  CpuGSEk<double, double>* g = static_cast<CpuGSEk<double, double>*>(h);
  const xyzq_t<double>* p = reinterpret_cast<const xyzq_t<double>*>(xyzq);
  g->spreadCharge1(n, p);
  g->solvePoisson();
  *energy = g->calculateEnergy();
  g->interpolateForce(n, p, fx, fy, fz);
  return 0;
}

void ref_gsek_destroy(void* h) { delete static_cast<CpuGSEk<double, double>*>(h); }

// CpuGaussCharge::spreadChargeToGrid for <double,double> (ct=0) and
// <double,float> (ct=1).
int ref_spread(int ct, int sx, int sy, int sz, double sigma, double rcut, int n, const void* xyzq,
               double boxx, double boxy, double boxz, int normalize, void* rho_out) {
  const size_t size = (size_t)sx * sy * sz;
  if (ct == 0) {
    CpuGaussCharge<double, double> gc(sx, sy, sz);
    CpuGrid<double> rho(sx, sy, sz);
    gc.spreadChargeToGrid(sigma, rcut, n, static_cast<const xyzq_t<double>*>(xyzq), boxx, boxy,
                          boxz, rho, normalize != 0);
    std::memcpy(rho_out, rho.getDataPointer(), size * sizeof(double));
  } else {
    CpuGaussCharge<double, float> gc(sx, sy, sz);
    CpuGrid<float> rho(sx, sy, sz);
    gc.spreadChargeToGrid(sigma, rcut, n, static_cast<const xyzq_t<float>*>(xyzq), boxx, boxy,
                          boxz, rho, normalize != 0);
    std::memcpy(rho_out, rho.getDataPointer(), size * sizeof(float));
  }
  return 0;
}

// CpuGaussCharge::interpolateForce (no ccelec factor) for <double,double>
// (ct=0) and <double,float> (ct=1).
int ref_gather(int ct, int sx, int sy, int sz, double sigma, double rcut, int n, const void* xyzq,
               double boxx, double boxy, double boxz, const void* phi_in, double* fx, double* fy,
               double* fz) {
  const size_t size = (size_t)sx * sy * sz;
  if (ct == 0) {
    CpuGaussCharge<double, double> gc(sx, sy, sz);
    CpuGrid<double> phi(sx, sy, sz);
    std::memcpy(phi.getDataPointer(), phi_in, size * sizeof(double));
    gc.interpolateForce(sigma, rcut, n, static_cast<const xyzq_t<double>*>(xyzq), boxx, boxy,
                        boxz, phi, fx, fy, fz);
  } else {
    CpuGaussCharge<double, float> gc(sx, sy, sz);
    CpuGrid<float> phi(sx, sy, sz);
    std::memcpy(phi.getDataPointer(), phi_in, size * sizeof(float));
    gc.interpolateForce(sigma, rcut, n, static_cast<const xyzq_t<float>*>(xyzq), boxx, boxy,
                        boxz, phi, fx, fy, fz);
  }
  return 0;
}

// CpuGaussCharge::spreadChargeOnGrid for <double,double> (ct=0) and
// <double,float> (ct=1).
int ref_spread_on_grid(int ct, int sx, int sy, int sz, double sigma, double rcut, double boxx,
                       double boxy, double boxz, const void* rho_in, void* rhoS_out) {
  const size_t size = (size_t)sx * sy * sz;
  if (ct == 0) {
    CpuGaussCharge<double, double> gc(sx, sy, sz);
    CpuGrid<double> rho(sx, sy, sz), rhoS(sx, sy, sz);
    std::memcpy(rho.getDataPointer(), rho_in, size * sizeof(double));
    gc.spreadChargeOnGrid(sigma, rcut, boxx, boxy, boxz, rho, rhoS);
    std::memcpy(rhoS_out, rhoS.getDataPointer(), size * sizeof(double));
  } else {
    CpuGaussCharge<double, float> gc(sx, sy, sz);
    CpuGrid<float> rho(sx, sy, sz), rhoS(sx, sy, sz);
    std::memcpy(rho.getDataPointer(), rho_in, size * sizeof(float));
    gc.spreadChargeOnGrid(sigma, rcut, boxx, boxy, boxz, rho, rhoS);
    std::memcpy(rhoS_out, rhoS.getDataPointer(), size * sizeof(float));
  }
  return 0;
}

// CpuGaussCharge::calcElectricFieldOnGrid, ct as above.
int ref_efield(int ct, int sx, int sy, int sz, double boxx, double boxy, double boxz,
               const void* phi_in, void* ex, void* ey, void* ez) {
  const size_t size = (size_t)sx * sy * sz;
  if (ct == 0) {
    CpuGaussCharge<double, double> gc(sx, sy, sz);
    CpuGrid<double> phi(sx, sy, sz), Ex(sx, sy, sz), Ey(sx, sy, sz), Ez(sx, sy, sz);
    std::memcpy(phi.getDataPointer(), phi_in, size * sizeof(double));
    gc.calcElectricFieldOnGrid(boxx, boxy, boxz, phi, Ex, Ey, Ez);
    std::memcpy(ex, Ex.getDataPointer(), size * sizeof(double));
    std::memcpy(ey, Ey.getDataPointer(), size * sizeof(double));
    std::memcpy(ez, Ez.getDataPointer(), size * sizeof(double));
  } else {
    CpuGaussCharge<double, float> gc(sx, sy, sz);
    CpuGrid<float> phi(sx, sy, sz), Ex(sx, sy, sz), Ey(sx, sy, sz), Ez(sx, sy, sz);
    std::memcpy(phi.getDataPointer(), phi_in, size * sizeof(float));
    gc.calcElectricFieldOnGrid(boxx, boxy, boxz, phi, Ex, Ey, Ez);
    std::memcpy(ex, Ex.getDataPointer(), size * sizeof(float));
    std::memcpy(ey, Ey.getDataPointer(), size * sizeof(float));
    std::memcpy(ez, Ez.getDataPointer(), size * sizeof(float));
  }
  return 0;
}

// CpuGaussCharge::calcDipoleSum, ct as above; dip receives (x, y, z).
int ref_dipole(int ct, int sx, int sy, int sz, double boxx, double boxy, double boxz,
               const void* rho_in, double* dip) {
  const size_t size = (size_t)sx * sy * sz;
  if (ct == 0) {
    CpuGaussCharge<double, double> gc(sx, sy, sz);
    CpuGrid<double> rho(sx, sy, sz);
    std::memcpy(rho.getDataPointer(), rho_in, size * sizeof(double));
    gc.calcDipoleSum(boxx, boxy, boxz, rho, dip[0], dip[1], dip[2]);
  } else {
    CpuGaussCharge<double, float> gc(sx, sy, sz);
    CpuGrid<float> rho(sx, sy, sz);
    std::memcpy(rho.getDataPointer(), rho_in, size * sizeof(float));
    gc.calcDipoleSum(boxx, boxy, boxz, rho, dip[0], dip[1], dip[2]);
  }
  return 0;
}

// CpuGreensFuncGSE<double>::mul on an interleaved half spectrum.
int ref_green_mul_d(int nx, int ny, int nz, double boxx, double boxy, double boxz, double sigma,
                    double* rhoK) {
  CpuGreensFuncGSE<double> g;
  CpuGrid<double> k((nx / 2 + 1) * 2, ny, nz);
  const size_t size = (size_t)(nx / 2 + 1) * 2 * ny * nz;
  std::memcpy(k.getDataPointer(), rhoK, size * sizeof(double));
  g.mul(nx, ny, nz, boxx, boxy, boxz, sigma, k);
  std::memcpy(rhoK, k.getDataPointer(), size * sizeof(double));
  return 0;
}

double ref_ewald_recip(double sigma, int kcut, double boxx, double boxy, double boxz,
                       double ccelec, int n, const double* xyzq, double* fx, double* fy,
                       double* fz) {
  CpuEwaldRecip e(sigma, kcut, boxx, boxy, boxz, ccelec);
  return e.calcForceEnergy(n, reinterpret_cast<const xyzq_t<double>*>(xyzq), fx, fy, fz);
}

double ref_ewald_direct(double sigma, double rcut, double boxx, double boxy, double boxz,
                        double ccelec, int n, const double* xyzq, int n_iblo14,
                        const int* iblo14, const int* inb14, double* fx, double* fy,
                        double* fz) {
  CpuEwaldDirect e(sigma, rcut, boxx, boxy, boxz, ccelec);
  if (n_iblo14 > 0) e.setupExclusions(n_iblo14, iblo14, inb14);
  return e.calcForceEnergy(n, reinterpret_cast<const xyzq_t<double>*>(xyzq), fx, fy, fz);
}

// CpuGrid<T>::save (CpuGrid.h:76-90, header-only): the reference's own grid
// text writer on a grid holding `data` (x fastest); type 0 = double, 1 = float.
int ref_grid_save(int type, int sx, int sy, int sz, const void* data, const char* filename) {
  const size_t size = (size_t)sx * sy * sz;
  if (type == 0) {
    CpuGrid<double> g(sx, sy, sz);
    std::memcpy(g.getDataPointer(), data, size * sizeof(double));
    static_cast<const CpuGrid<double>&>(g).save(filename);
  } else {
    CpuGrid<float> g(sx, sy, sz);
    std::memcpy(g.getDataPointer(), data, size * sizeof(float));
    static_cast<const CpuGrid<float>&>(g).save(filename);
  }
  return 0;
}

}  // extern "C"
