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

}  // namespace gse
