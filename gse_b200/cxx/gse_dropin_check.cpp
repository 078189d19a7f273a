// gse_dropin_check.cpp -- a caller written against the reference's class API
// (the sequence cpu_gse.cpp runs for its GSE-k test, cpu_gse.cpp:424-455),
// compiled against gse_dropin.h instead of the reference headers.
//
// usage: gse_dropin_check fp64|mixed Mx My Mz Lx Ly Lz sigma xyzq.txt
//   xyzq.txt: one "x y z q" record per line.
// Prints "E <energy>" and one "F fx fy fz" line per atom from CpuGSEk, then
// "E_stages <energy>" and "F_stages ..." lines from the same computation
// assembled out of CpuGaussCharge, CpuGreensFuncGSE and CpuFFTSolver.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "gse_dropin.h"

using gse_b200::CpuEwaldDirect;
using gse_b200::CpuEwaldRecip;
using gse_b200::CpuFFTSolver;
using gse_b200::CpuGaussCharge;
using gse_b200::CpuGreensFuncGSE;
using gse_b200::CpuGrid;
using gse_b200::CpuGSEk;
using gse_b200::xyzq_t;

template <typename CT>
int run(int M[3], double L[3], double sigma, const std::vector<double>& raw) {
  const int n = (int)raw.size() / 4;
  std::vector<xyzq_t<CT>> xyzq(n);
  for (int i = 0; i < n; i++)
    xyzq[i] = {(CT)raw[4 * i], (CT)raw[4 * i + 1], (CT)raw[4 * i + 2], (CT)raw[4 * i + 3]};
  const double kappa = 0.4, lambdaSigma = 3.0, lambdaSigma1 = 3.0, ccelec = 332.0716;
  std::vector<double> fx(n), fy(n), fz(n);

  CpuGSEk<double, CT> gse(M[0], M[1], M[2], sigma, kappa, lambdaSigma, lambdaSigma1, L[0], L[1],
                          L[2], ccelec);
  gse.spreadCharge1(n, xyzq.data());
  gse.solvePoisson();
  const double E = gse.calculateEnergy();
  gse.interpolateForce(n, xyzq.data(), fx.data(), fy.data(), fz.data());
  int paths = 0;
  gse_b200::check(gse_get_paths(gse.context(), &paths));
  printf("PATHS %d\n", paths);
  printf("E %.17g\n", E);
  for (int i = 0; i < n; i++) printf("F %.17g %.17g %.17g\n", fx[i], fy[i], fz[i]);

  // the same evaluation from the stage classes
  const double sigma1 = gse.getSigma1(), sigma2 = gse.getSigma2();
  const double rcut = gse.getLambdaSigma1() * std::sqrt(2.0) * sigma1;
  CpuGaussCharge<double, CT> gauss(M[0], M[1], M[2]);
  CpuGreensFuncGSE<CT> green;
  CpuFFTSolver<CT> solver(green, M[0], M[1], M[2]);
  CpuGrid<CT> rho(M[0], M[1], M[2]), phi(M[0], M[1], M[2]);
  gauss.spreadChargeToGrid(sigma1, rcut, n, xyzq.data(), L[0], L[1], L[2], rho);
  solver.run(phi, rho, sigma2, L[0], L[1], L[2]);
  double dot = 0.0;
  for (int i = 0; i < rho.getSize(); i++)
    dot += (double)rho.getDataPointer()[i] * (double)phi.getDataPointer()[i];
  const double h3 = (L[0] / M[0]) * (L[1] / M[1]) * (L[2] / M[2]);
  printf("E_stages %.17g\n", 0.5 * ccelec * h3 * dot);
  gauss.interpolateForce(sigma1, rcut, n, xyzq.data(), L[0], L[1], L[2], phi, fx.data(),
                         fy.data(), fz.data());
  for (int i = 0; i < n; i++)
    printf("F_stages %.17g %.17g %.17g\n", ccelec * fx[i], ccelec * fy[i], ccelec * fz[i]);

  // the real-space variant's second spreading step (CpuGSEr::spreadCharge2)
  // and the grid field and dipole of the first spreading
  if (getenv("GSE_CHECK_GRID_OPS")) {
    const double rcut2 = gse.getLambdaSigma1() * std::sqrt(2.0) * sigma2;
    CpuGrid<CT> rhoS(M[0], M[1], M[2]), Ex(M[0], M[1], M[2]), Ey(M[0], M[1], M[2]),
        Ez(M[0], M[1], M[2]);
    gauss.spreadChargeOnGrid(sigma2, rcut2, L[0], L[1], L[2], rho, rhoS);
    gauss.calcElectricFieldOnGrid(L[0], L[1], L[2], phi, Ex, Ey, Ez);
    double dip[3];
    gauss.calcDipoleSum(L[0], L[1], L[2], rho, dip[0], dip[1], dip[2]);
    printf("DIP %.17g %.17g %.17g\n", dip[0], dip[1], dip[2]);
    for (int i = 0; i < rho.getSize(); i++)
      printf("G %.17g %.17g %.17g %.17g %.17g %.17g\n", (double)rho.getDataPointer()[i],
             (double)phi.getDataPointer()[i], (double)rhoS.getDataPointer()[i],
             (double)Ex.getDataPointer()[i], (double)Ey.getDataPointer()[i],
             (double)Ez.getDataPointer()[i]);
  }
  // the reference's third instance, CpuGaussCharge<float,float>
  // (CpuGaussCharge.cpp:524-526): the same spread, then the gather from the
  // solved potential with float force arrays
  if constexpr (std::is_same<CT, float>::value) {
    if (getenv("GSE_CHECK_FLOAT_FLOAT")) {
      CpuGaussCharge<float, float> gff(M[0], M[1], M[2]);
      CpuGrid<float> rff(M[0], M[1], M[2]);
      gff.spreadChargeToGrid(sigma1, rcut, n, xyzq.data(), L[0], L[1], L[2], rff);
      for (int i = 0; i < rff.getSize(); i++) printf("RFF %.9g\n", rff.getDataPointer()[i]);
      std::vector<float> gx(n), gy(n), gz(n);
      gff.interpolateForce(sigma1, rcut, n, xyzq.data(), L[0], L[1], L[2], phi, gx.data(),
                           gy.data(), gz.data());
      for (int i = 0; i < n; i++) printf("FFF %.9g %.9g %.9g\n", gx[i], gy[i], gz[i]);
      for (int i = 0; i < phi.getSize(); i++) printf("PHI %.9g\n", phi.getDataPointer()[i]);
    }
  }
  // the FP64 Ewald references of the same charges (the sequence of
  // cpu_gse.cpp:555-560), with the water exclusions of rigid 3-site molecules
  if (getenv("GSE_CHECK_EWALD")) {
    std::vector<xyzq_t<double>> x64(n);
    for (int i = 0; i < n; i++)
      x64[i] = {raw[4 * i], raw[4 * i + 1], raw[4 * i + 2], raw[4 * i + 3]};
    std::vector<int> iblo14(n), inb14;
    for (int a = 0; a < n; a++) {
      const int m0 = a - a % 3;
      if (m0 + 2 < n)
        for (int b = a + 1; b < m0 + 3; b++) inb14.push_back(b + 1);
      iblo14[a] = (int)inb14.size();
    }
    CpuEwaldRecip rec(sigma, 12, L[0], L[1], L[2]);
    const double er = rec.calcForceEnergy(n, x64.data(), fx.data(), fy.data(), fz.data());
    printf("EWR %.17g\n", er);
    for (int i = 0; i < n; i++) printf("FWR %.17g %.17g %.17g\n", fx[i], fy[i], fz[i]);
    CpuEwaldDirect dir(sigma, 9.0, L[0], L[1], L[2]);
    dir.setupExclusions(n, iblo14.data(), inb14.data());
    const double ed = dir.calcForceEnergy(n, x64.data(), fx.data(), fy.data(), fz.data());
    printf("EWD %.17g\n", ed);
    for (int i = 0; i < n; i++) printf("FWD %.17g %.17g %.17g\n", fx[i], fy[i], fz[i]);
  }
  return 0;
}

int main(int argc, char** argv) {
  if (argc != 10) {
    fprintf(stderr, "usage: %s fp64|mixed Mx My Mz Lx Ly Lz sigma xyzq.txt\n", argv[0]);
    return 2;
  }
  int M[3] = {atoi(argv[2]), atoi(argv[3]), atoi(argv[4])};
  double L[3] = {atof(argv[5]), atof(argv[6]), atof(argv[7])};
  const double sigma = atof(argv[8]);
  FILE* f = fopen(argv[9], "r");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", argv[9]);
    return 2;
  }
  std::vector<double> raw;
  double v;
  while (fscanf(f, "%lf", &v) == 1) raw.push_back(v);
  fclose(f);
  try {
    if (!strcmp(argv[1], "fp64")) return run<double>(M, L, sigma, raw);
    if (!strcmp(argv[1], "mixed")) return run<float>(M, L, sigma, raw);
    fprintf(stderr, "precision must be fp64 or mixed\n");
    return 2;
  } catch (const gse_b200::Error& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
