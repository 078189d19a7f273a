// gse_dropin.h -- C++ classes with the reference's GSE-k API, running on the
// B200 through the C ABI of libgse_b200.so (include/gse_b200.h).
//
// Each class keeps the constructor and method signatures of its reference
// counterpart (paths relative to ap-hynninen/GSE):
//
//   xyzq_t<T>                  TypesGSE.h:19-22
//   CpuGrid<T>                 Grid.h:12-55, CpuGrid.h:17-108 (host container)
//   CpuGaussCharge<AT,CT>      CpuGaussCharge.h:11-49 (<double,double>, <double,float>,
//                              <float,float>)
//   CpuGreensFunc<T>           CpuGreensFunc.h:10-19
//   CpuGreensFuncGSE<T>        CpuGreensFuncGSE.h:10-19
//   CpuFFTSolver<T>            CpuFFTSolver.h:12-42
//   CpuGSE<AT,CT>, CpuGSEk     CpuGSE.h:19-68, CpuGSEk.h:19-37
//   CpuEwaldRecip              CpuEwaldRecip.h:11-44 (calcForceEnergy, FP64)
//   CpuEwaldDirect             CpuEwaldDirect.h:10-44 (FP64)
//   Erms, loadArray, saveForce, readForce   cpu_gse.cpp:128-196 (driver text I/O)
//
// so that a caller switches by including this header instead of the
// reference's and bringing the names into scope (`using namespace gse_b200;`
// or one using-declaration per class).  Instances: <double,double> is the
// plain FP64 form, <double,float> the mixed form.
//
// Differences a caller can see:
//  - where the reference asserts or calls exit(), these classes throw
//    gse_b200::Error (status code + message);
//  - CpuFFTSolver takes only the GSE Green's function (the only one on the
//    path); any other CpuGreensFunc is rejected at construction;
//  - the grids returned by getRhoS()/getPhi() are host copies refreshed on
//    each call, so the results live on the GPU until a caller asks for them.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "gse_b200.h"

namespace gse_b200 {

class Error : public std::runtime_error {
 public:
  Error(gse_status_t s, const std::string& what)
      : std::runtime_error(std::string(gse_status_string(s)) + ": " + what), status(s) {}
  gse_status_t status;
};

inline void check(gse_status_t s) {
  if (s != GSE_OK) throw Error(s, gse_last_error());
}

template <typename T>
struct xyzq_t {
  T x, y, z, q;
};

template <typename T>
constexpr int precision_of() {
  static_assert(std::is_same<T, double>::value || std::is_same<T, float>::value,
                "calculation type must be double or float");
  return std::is_same<T, double>::value ? GSE_PRECISION_FP64 : GSE_PRECISION_MIXED;
}

// RAII owner of one gse_context_t.
class Context {
 public:
  Context(int sx, int sy, int sz, double sigma, double kappa, double lambdaSigma,
          double lambdaSigma1, double bx, double by, double bz, double ccelec, int precision,
          int device = 0) {
    gse_params_t p;
    gse_params_default(&p);
    p.size_x = sx;
    p.size_y = sy;
    p.size_z = sz;
    p.sigma = sigma;
    p.kappa = kappa;
    p.lambda_sigma = lambdaSigma;
    p.lambda_sigma1 = lambdaSigma1;
    p.box_x = bx;
    p.box_y = by;
    p.box_z = bz;
    p.ccelec = ccelec;
    p.precision = precision;
    p.device = device;
    check(gse_create(&p, &ctx_));
  }
  ~Context() { gse_destroy(ctx_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  gse_context_t* get() const { return ctx_; }

 private:
  gse_context_t* ctx_ = nullptr;
};

// ---------------------------------------------------------------------------
// Grid<T> / CpuGrid<T>: x-fastest periodic host grid.
// ---------------------------------------------------------------------------
template <typename T>
class CpuGrid {
 public:
  CpuGrid(const int sizeX, const int sizeY, const int sizeZ)
      : sizeX(sizeX), sizeY(sizeY), sizeZ(sizeZ), size(sizeX * sizeY * sizeZ),
        data_((size_t)sizeX * sizeY * sizeZ, T(0)) {}

  T* getDataPointer() { return data_.data(); }
  const T* getDataPointer() const { return data_.data(); }
  int getPos(const int x, const int y, const int z) const {
    const int xt = (x + sizeX) % sizeX, yt = (y + sizeY) % sizeY, zt = (z + sizeZ) % sizeZ;
    return xt + (yt + zt * sizeY) * sizeX;
  }
  int getSizeX() const { return sizeX; }
  int getSizeY() const { return sizeY; }
  int getSizeZ() const { return sizeZ; }
  int getSize() const { return size; }

  void clear() { std::fill(data_.begin(), data_.end(), T(0)); }
  template <typename T2>
  void add(const CpuGrid<T2>& g) {
    const T2* d = g.getDataPointer();
    for (int i = 0; i < size; i++) data_[i] += (T)d[i];
  }
  template <typename T2>
  void sub(const CpuGrid<T2>& g) {
    const T2* d = g.getDataPointer();
    for (int i = 0; i < size; i++) data_[i] -= (T)d[i];
  }
  template <typename T2>
  void copy(const CpuGrid<T2>& g) {
    const T2* d = g.getDataPointer();
    for (int i = 0; i < size; i++) data_[i] = (T)d[i];
  }
  void scale(const T val) {
    for (T& v : data_) v *= val;
  }
  T sum() const {
    T r = T(0);
    for (T v : data_) r += v;
    return r;
  }
  T maxAbsValue() const {
    T m = T(0);
    for (T v : data_) m = std::fabs(v) > m ? std::fabs(v) : m;
    return m;
  }
  T getDataValue(const int x, const int y, const int z) const { return data_[getPos(x, y, z)]; }
  // One value per line, z outermost (CpuGrid.h:76-106); throws instead of exit(1).
  void save(const char* filename) const {
    std::ofstream f(filename);
    if (!f.is_open())
      throw Error(GSE_ERR_INVALID_ARG, std::string("CpuGrid::save, cannot open ") + filename);
    for (int i = 0; i < size; i++) f << data_[i] << "\n";
  }

  const int sizeX, sizeY, sizeZ, size;

 private:
  std::vector<T> data_;
};

// ---------------------------------------------------------------------------
// CpuGaussCharge<AT,CT>: spreading and interpolation with explicit sigma,
// cut-off and box (CpuGaussCharge.cpp:105-384), and the grid operations
// beside them (CpuGaussCharge.cpp:62-98, :188-226, :390-519).
// ---------------------------------------------------------------------------
template <typename AT, typename CT>
class CpuGaussCharge {
  // the reference's instances (CpuGaussCharge.cpp:524-526): <double,double>,
  // <double,float> and <float,float>; with AT = float the forces and the
  // dipole are accumulated in double on the GPU and rounded to float once
  static_assert(std::is_same<AT, double>::value ||
                    (std::is_same<AT, float>::value && std::is_same<CT, float>::value),
                "instances: <double,double>, <double,float>, <float,float>");

 public:
  // The stage calls carry their own sigma, cut-off and box; the context's
  // own parameters only have to describe a valid stencil.
  CpuGaussCharge(const int sizeX, const int sizeY, const int sizeZ)
      : sizeX(sizeX), sizeY(sizeY), sizeZ(sizeZ),
        ctx_(sizeX, sizeY, sizeZ, 1.0, 0.4, 3.0, 3.0, sizeX, sizeY, sizeZ, 332.0716,
             precision_of<CT>()) {}

  // Number of offsets with r^2 < rcut^2 (CpuGaussCharge.cpp:28-56): the
  // spacings and rcut^2 rounded to CT, the distances formed and summed in CT.
  int calcSupportSize(const double rcut, const double boxx, const double boxy,
                      const double boxz) const {
    const double hd[3] = {boxx / sizeX, boxy / sizeY, boxz / sizeZ};
    int n[3];
    CT h[3];
    for (int d = 0; d < 3; d++) {
      n[d] = (int)std::ceil(rcut / hd[d]);
      h[d] = (CT)hd[d];
    }
    const CT rcut2 = (CT)(rcut * rcut);
    int cnt = 0;
    for (int tz = -n[2]; tz <= n[2]; tz++) {
      const CT dz = ((CT)(std::abs(tz) - 1)) * h[2];
      for (int ty = -n[1]; ty <= n[1]; ty++) {
        const CT dy = ((CT)(std::abs(ty) - 1)) * h[1];
        for (int tx = -n[0]; tx <= n[0]; tx++) {
          const CT dx = ((CT)(std::abs(tx) - 1)) * h[0];
          const CT r2 = dx * dx + dy * dy + dz * dz;
          if (r2 < rcut2) cnt++;
        }
      }
    }
    return cnt;
  }

  void spreadChargeToGrid(const double sigma, const double rcut, const int numCoord,
                          const xyzq_t<CT>* xyzq, const double boxx, const double boxy,
                          const double boxz, CpuGrid<CT>& rho, const bool normalize = false) {
    same_size(rho);
    check(gse_gauss_spread(ctx_.get(), sigma, rcut, numCoord, xyzq, boxx, boxy, boxz,
                           normalize ? 1 : 0, rho.getDataPointer()));
  }

  void interpolateForce(const double sigma, const double rcut, const int numCoord,
                        const xyzq_t<CT>* xyzq, const double boxx, const double boxy,
                        const double boxz, const CpuGrid<CT>& phi, AT* forceX, AT* forceY,
                        AT* forceZ) {
    same_size(phi);
    if constexpr (std::is_same<AT, double>::value) {
      check(gse_gauss_interpolate(ctx_.get(), sigma, rcut, numCoord, xyzq, boxx, boxy, boxz,
                                  phi.getDataPointer(), forceX, forceY, forceZ));
    } else {
      const size_t n = numCoord > 0 ? (size_t)numCoord : 0;
      std::vector<double> f(3 * n);
      check(gse_gauss_interpolate(ctx_.get(), sigma, rcut, numCoord, xyzq, boxx, boxy, boxz,
                                  phi.getDataPointer(), f.data(), f.data() + n,
                                  f.data() + 2 * n));
      for (size_t i = 0; i < n; i++) {
        forceX[i] = (AT)f[i];
        forceY[i] = (AT)f[n + i];
        forceZ[i] = (AT)f[2 * n + i];
      }
    }
  }

  // On-grid Gaussian convolution, rhoS = G(sigma) * rho (CpuGaussCharge.cpp:390-519).
  void spreadChargeOnGrid(const double sigma, const double rcut, const double boxx,
                          const double boxy, const double boxz, const CpuGrid<CT>& rho,
                          CpuGrid<CT>& rhoS) {
    same_size(rho);
    same_size(rhoS);
    check(gse_gauss_spread_on_grid(ctx_.get(), sigma, rcut, boxx, boxy, boxz,
                                   rho.getDataPointer(), rhoS.getDataPointer()));
  }

  // Forward-difference field on the grid (CpuGaussCharge.cpp:62-98).
  void calcElectricFieldOnGrid(const double boxx, const double boxy, const double boxz,
                               const CpuGrid<CT>& phi, CpuGrid<CT>& Ex, CpuGrid<CT>& Ey,
                               CpuGrid<CT>& Ez) {
    same_size(phi);
    same_size(Ex);
    same_size(Ey);
    same_size(Ez);
    check(gse_gauss_efield_on_grid(ctx_.get(), boxx, boxy, boxz, phi.getDataPointer(),
                                   Ex.getDataPointer(), Ey.getDataPointer(),
                                   Ez.getDataPointer()));
  }

  // Dipole sum of a charge grid (CpuGaussCharge.cpp:188-226).
  void calcDipoleSum(const double boxx, const double boxy, const double boxz,
                     const CpuGrid<CT>& rho, AT& dipSumX, AT& dipSumY, AT& dipSumZ) {
    same_size(rho);
    double d[3];
    check(gse_gauss_dipole_sum(ctx_.get(), boxx, boxy, boxz, rho.getDataPointer(), d));
    dipSumX = d[0];
    dipSumY = d[1];
    dipSumZ = d[2];
  }

 private:
  template <typename G>
  void same_size(const G& g) const {
    if (g.getSizeX() != sizeX || g.getSizeY() != sizeY || g.getSizeZ() != sizeZ)
      throw Error(GSE_ERR_INVALID_ARG, "grid size mismatch (CpuGaussCharge.cpp:240-242)");
  }
  const int sizeX, sizeY, sizeZ;
  Context ctx_;
};

// ---------------------------------------------------------------------------
// Green's functions and the FFT solver.
// ---------------------------------------------------------------------------
template <typename T>
class CpuGreensFunc {
 public:
  virtual ~CpuGreensFunc() {}
  virtual void mul(const int nfftX, const int nfftY, const int nfftZ, const double boxx,
                   const double boxy, const double boxz, const double sigma,
                   CpuGrid<T>& rho) = 0;
};

// k-space GSE Green's function.  rho is the half spectrum as interleaved
// complex values: a CpuGrid of ((nfftX/2+1)*2, nfftY, nfftZ) reals.
template <typename T>
class CpuGreensFuncGSE : public CpuGreensFunc<T> {
 public:
  void mul(const int nfftX, const int nfftY, const int nfftZ, const double boxx,
           const double boxy, const double boxz, const double sigma, CpuGrid<T>& rho) override {
    if ((nfftX / 2 + 1) * 2 != rho.getSizeX() || nfftY != rho.getSizeY() ||
        nfftZ != rho.getSizeZ())
      throw Error(GSE_ERR_INVALID_ARG, "k-space grid size mismatch (CpuGreensFuncGSE.cpp:13-15)");
    if (!ctx_ || M_[0] != nfftX || M_[1] != nfftY || M_[2] != nfftZ) {
      ctx_.reset();
      ctx_.reset(new Context(nfftX, nfftY, nfftZ, 1.0, 0.4, 3.0, 3.0, nfftX, nfftY, nfftZ,
                             332.0716, precision_of<T>()));
      M_[0] = nfftX;
      M_[1] = nfftY;
      M_[2] = nfftZ;
    }
    check(gse_green_mul(ctx_->get(), sigma, boxx, boxy, boxz, rho.getDataPointer()));
  }

 private:
  std::unique_ptr<Context> ctx_;
  int M_[3] = {0, 0, 0};
};

template <typename T>
class CpuFFTSolver {
 public:
  CpuFFTSolver(CpuGreensFunc<T>& greensFunc, const int sizeX, const int sizeY, const int sizeZ)
      : sizeX(sizeX), sizeY(sizeY), sizeZ(sizeZ), gse_(check_gse(greensFunc)),
        ctx_(sizeX, sizeY, sizeZ, 1.0, 0.4, 3.0, 3.0, sizeX, sizeY, sizeZ, 332.0716,
             precision_of<T>()) {}

  // phi = c2r(G(sigma) r2c(rho)) (CpuFFTSolver.cpp:75-96).
  void run(CpuGrid<T>& phi, const CpuGrid<T>& rho, const double sigma, const double boxx,
           const double boxy, const double boxz) {
    const CpuGrid<T>* grids[2] = {&phi, &rho};
    for (const CpuGrid<T>* g : grids)
      if (g->getSizeX() != sizeX || g->getSizeY() != sizeY || g->getSizeZ() != sizeZ)
        throw Error(GSE_ERR_INVALID_ARG, "grid size mismatch (CpuFFTSolver.cpp:78-83)");
    check(gse_fft_solve(ctx_.get(), sigma, boxx, boxy, boxz, rho.getDataPointer(),
                        phi.getDataPointer()));
  }

 private:
  static CpuGreensFuncGSE<T>* check_gse(CpuGreensFunc<T>& g) {
    CpuGreensFuncGSE<T>* p = dynamic_cast<CpuGreensFuncGSE<T>*>(&g);
    if (!p)
      throw Error(GSE_ERR_UNSUPPORTED, "only the GSE Green's function is implemented on the GPU");
    return p;
  }
  const int sizeX, sizeY, sizeZ;
  CpuGreensFuncGSE<T>* gse_;
  Context ctx_;
};

// ---------------------------------------------------------------------------
// CpuGSE<AT,CT> and CpuGSEk<AT,CT>.
// ---------------------------------------------------------------------------
template <typename AT, typename CT>
class CpuGSE {
  static_assert(std::is_same<AT, double>::value, "forces and energies are accumulated in double");

 public:
  CpuGSE(const int sizeX, const int sizeY, const int sizeZ, const double sigma,
         const double kappa, const double lambdaSigma, const double lambdaSigma1,
         const double boxx, const double boxy, const double boxz, const double ccelec = 332.0716)
      : ccelec(ccelec), boxx(boxx), boxy(boxy), boxz(boxz), sigma(sigma), kappa(kappa),
        lambdaSigma(lambdaSigma), lambdaSigma1(lambdaSigma1),
        sigma1(sigma * std::sqrt(kappa)), sigma2(sigma * std::sqrt(1.0 - 2.0 * kappa)),
        rhoS(sizeX, sizeY, sizeZ), phiM(sizeX, sizeY, sizeZ),
        ctx_(sizeX, sizeY, sizeZ, sigma, kappa, lambdaSigma, lambdaSigma1, boxx, boxy, boxz,
             ccelec, precision_of<CT>()) {}
  virtual ~CpuGSE() {}

  void printInfo() {
    printf("sizeX=%d sizeY=%d sizeZ=%d\n", rhoS.getSizeX(), rhoS.getSizeY(), rhoS.getSizeZ());
    printf("sigma=%g sigma1=%g sigma2=%g kappa=%g\n", sigma, sigma1, sigma2, kappa);
    printf("lambdaSigma1=%g lambdaSigma=%g\n", lambdaSigma1, lambdaSigma);
  }
  void setBoxSize(const double bx, const double by, const double bz) {
    check(gse_set_box(ctx_.get(), bx, by, bz));
    boxx = bx;
    boxy = by;
    boxz = bz;
  }
  virtual void spreadCharge1(const int numCoord, const xyzq_t<CT>* xyzq) = 0;
  virtual void solvePoisson() = 0;
  virtual AT calculateEnergy() = 0;
  void interpolateForce(const int numCoord, const xyzq_t<CT>* xyzq, AT* forceX, AT* forceY,
                        AT* forceZ) {
    check(gse_interpolate_force(ctx_.get(), numCoord, xyzq, forceX, forceY, forceZ));
  }
  CpuGrid<CT>& getRhoS() {
    check(gse_get_grid(ctx_.get(), GSE_GRID_RHO, rhoS.getDataPointer()));
    return rhoS;
  }
  CpuGrid<CT>& getPhi() {
    check(gse_get_grid(ctx_.get(), GSE_GRID_PHI, phiM.getDataPointer()));
    return phiM;
  }
  // Electric field at the atoms (force per unit charge, times ccelec) from
  // phiM; the reference's interpolation loop serves force and field alike.
  void interpolateField(const int numCoord, const xyzq_t<CT>* xyzq, AT* fieldX, AT* fieldY,
                        AT* fieldZ) {
    check(gse_interpolate_field(ctx_.get(), numCoord, xyzq, fieldX, fieldY, fieldZ));
  }
  // Reciprocal-space virial of the current rhoS (xx, yy, zz, xy, xz, yz); the
  // reference classes compute none (gse_virial).
  void calculateVirial(double virial[6]) { check(gse_virial(ctx_.get(), virial)); }
  double getSigma1() { return sigma1; }
  double getSigma2() { return sigma2; }
  double getLambdaSigma1() { return lambdaSigma1; }
  // Not in the reference: the underlying context, for gse_* calls.
  gse_context_t* context() { return ctx_.get(); }

 protected:
  const double ccelec;
  double boxx, boxy, boxz;
  double sigma, kappa, lambdaSigma, lambdaSigma1, sigma1, sigma2;
  CpuGrid<CT> rhoS, phiM;
  Context ctx_;
};

template <typename AT, typename CT>
class CpuGSEk : public CpuGSE<AT, CT> {
 public:
  CpuGSEk(const int sizeX, const int sizeY, const int sizeZ, const double sigma,
          const double kappa, const double lambdaSigma, const double lambdaSigma1,
          const double boxx, const double boxy, const double boxz, const double ccelec = 332.0716)
      : CpuGSE<AT, CT>(sizeX, sizeY, sizeZ, sigma, kappa, lambdaSigma, lambdaSigma1, boxx, boxy,
                       boxz, ccelec) {}
  void spreadCharge1(const int numCoord, const xyzq_t<CT>* xyzq) override {
    check(gse_spread_charge(this->ctx_.get(), numCoord, xyzq));
  }
  void solvePoisson() override { check(gse_solve_poisson(this->ctx_.get())); }
  AT calculateEnergy() override {
    double e = 0.0;
    check(gse_calculate_energy(this->ctx_.get(), &e));
    return e;
  }
};

// ---------------------------------------------------------------------------
// Text I/O and the force error measure of the reference's driver
// (cpu_gse.cpp:128-198): the same formats (iostream defaults, one record per
// line), throwing gse_b200::Error where the reference calls exit(1).
// ---------------------------------------------------------------------------
// Relative RMS difference sqrt(sum |x - ref|^2 / sum |ref|^2) (cpu_gse.cpp:128-145).
inline double Erms(const int n, const double* refx, const double* refy, const double* refz,
                   const double* x, const double* y, const double* z) {
  double rms = 0.0, ref = 0.0;
  for (int i = 0; i < n; i++) {
    const double dx = x[i] - refx[i], dy = y[i] - refy[i], dz = z[i] - refz[i];
    rms += dx * dx + dy * dy + dz * dz;
    ref += refx[i] * refx[i] + refy[i] * refy[i] + refz[i] * refz[i];
  }
  return std::sqrt(rms / ref);
}

// numLine records of `width` whitespace-separated values (cpu_gse.cpp:150-170).
template <typename T>
void loadArray(const int width, const int numLine, const char* filename, T* array) {
  std::ifstream file(filename);
  if (!file.is_open())
    throw Error(GSE_ERR_INVALID_ARG, std::string("cannot open ") + filename);
  for (int i = 0; i < numLine * width; i++)
    if (!(file >> array[i]))
      throw Error(GSE_ERR_INVALID_ARG, std::string("error reading ") + filename);
}

// "fx fy fz" per line (cpu_gse.cpp:172-182).
template <typename T>
void saveForce(const char* filename, const int numCoord, const T* forceX, const T* forceY,
               const T* forceZ) {
  std::ofstream file(filename);
  if (!file.is_open())
    throw Error(GSE_ERR_INVALID_ARG, std::string("cannot open ") + filename);
  for (int i = 0; i < numCoord; i++)
    file << forceX[i] << " " << forceY[i] << " " << forceZ[i] << "\n";
}

// The file saveForce writes (cpu_gse.cpp:185-196).
template <typename T>
void readForce(const char* filename, const int numCoord, T* forceX, T* forceY, T* forceZ) {
  std::ifstream file(filename);
  if (!file.is_open())
    throw Error(GSE_ERR_INVALID_ARG, std::string("cannot open ") + filename);
  for (int i = 0; i < numCoord; i++)
    if (!(file >> forceX[i] >> forceY[i] >> forceZ[i]))
      throw Error(GSE_ERR_INVALID_ARG, std::string("error reading ") + filename);
}

// The FP64 Ewald sums, the accuracy references of the GSE-k forms.  Their
// arrays are host memory, as in the reference; each call returns with the
// results written.
class CpuEwaldRecip {
 public:
  CpuEwaldRecip(const double sigma, const int kcut, const double boxx_in, const double boxy_in,
                const double boxz_in, const double ccelec = 332.0716)
      : ccelec(ccelec), sigma(sigma), kcut(kcut) {
    setBoxsize(boxx_in, boxy_in, boxz_in);
  }
  // E over the k != 0 with |k|^2 <= kcut^2 and the force -dE/dx
  // (CpuEwaldRecip.cpp:87-147)
  double calcForceEnergy(const int n, const xyzq_t<double>* xyzq, double* fx, double* fy,
                         double* fz) {
    double e = 0.0;
    check(gse_ewald_recip(0, nullptr, sigma, kcut, boxx, boxy, boxz, ccelec, n,
                          reinterpret_cast<const double*>(xyzq), &e, fx, fy, fz));
    return e;
  }
  void setSigma(const double sigma_in) { sigma = sigma_in; }
  void setBoxsize(const double boxx_in, const double boxy_in, const double boxz_in) {
    boxx = boxx_in;
    boxy = boxy_in;
    boxz = boxz_in;
  }

 private:
  const double ccelec;
  double sigma;
  int kcut;
  double boxx, boxy, boxz;
};

class CpuEwaldDirect {
 public:
  CpuEwaldDirect(const double sigma, const double rcut, const double boxx, const double boxy,
                 const double boxz, const double ccelec = 332.0716)
      : ccelec(ccelec), sigma(sigma), rcut(rcut), boxx(boxx), boxy(boxy), boxz(boxz) {}
  // CHARMM exclusion lists (CpuEwaldDirect.cpp:31-40): iblo14[a] is the
  // cumulative end of atom a's 1-based partners in inb14
  void setupExclusions(const int n_iblo14_in, const int* iblo14_in, const int* inb14_in) {
    iblo14.assign(iblo14_in, iblo14_in + n_iblo14_in);
    const int n_inb14 = n_iblo14_in > 0 ? iblo14.back() : 0;
    inb14.assign(inb14_in, inb14_in + std::max(n_inb14, 0));
  }
  // E including the self energy, and the gradient dE/dx in fx, fy, fz, as
  // the reference's arrays hold it (CpuEwaldDirect.cpp:45-131)
  double calcForceEnergy(const int n, const xyzq_t<double>* xyzq, double* fx, double* fy,
                         double* fz) {
    double e = 0.0;
    check(gse_ewald_direct(0, nullptr, sigma, rcut, boxx, boxy, boxz, ccelec, n,
                           reinterpret_cast<const double*>(xyzq), (int)iblo14.size(),
                           iblo14.empty() ? nullptr : iblo14.data(),
                           inb14.empty() ? nullptr : inb14.data(), &e, fx, fy, fz));
    return e;
  }

 private:
  const double ccelec;
  double sigma, rcut, boxx, boxy, boxz;
  std::vector<int> iblo14, inb14;
};

}  // namespace gse_b200
