// gse_ewald.cuh -- FP64 Ewald reciprocal sum on the GPU (gse_ewald.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace gse {

struct EwGeom {
  double inv_box[3];
  double pref;          // 2 pi / V * ccelec
  double half_sigmasq;  // sigma^2 / 2
};

struct EwRowHost {
  int ky, kz, kx0, nk;
  long long off;
};

struct EwScratch {
  void* rows;          // [nrows] rows
  double2* S;          // [number of half-space k] P(k) S(k)
  double* row_energy;  // [nrows]
};

std::vector<EwRowHost> ewald_rows(int kcut);
cudaError_t launch_ewald(const double4* xyzq, int n, const std::vector<EwRowHost>& rows,
                         const EwGeom& g, EwScratch w, double* fx, double* fy, double* fz,
                         cudaStream_t st);

// ---- direct (real-space) sum, gse_ewald_direct.cu ----

constexpr int kEwdMaxCellsPerAxis = 128;

struct EwdGeom {
  double box[3], hbox[3], inv_box[3];
  int nc[3];  // cells per axis, each of side box / nc >= rcut
  int ncell;
  double rcut2, inv_sqrt2sigma, inv_2sigmasq, two_sqrtpi;
  double self;  // -ccelec / sqrt(2 pi sigma^2)
  double ccelec;
};

struct EwdScratch {
  int* key;         // [n] cell of each atom
  int* counts;      // [ncell]
  int* start;       // [ncell + 1]
  int* tile_sums;   // [ceil(ncell / 4096)]
  int* tmp;         // [n]
  double4* sorted;  // [n] atoms in cell order
  int* perm;        // [n] original index of each sorted atom
  double* partials; // [ncell] energy per cell
  unsigned* done;   // counter of finished cells
};

EwdGeom ewald_direct_geom(double sigma, double rcut, const double box[3], double ccelec);
// ex_start[n + 1] / ex_idx: the excluded partners of every atom (both
// directions), or both NULL.  energy_out: one device double.
cudaError_t launch_ewald_direct(const double4* xyzq, int n, const EwdGeom& g, EwdScratch w,
                                const int* ex_start, const int* ex_idx, double* fx, double* fy,
                                double* fz, double* energy_out, cudaStream_t st);

}  // namespace gse
