// gse_kernels.cuh -- launcher declarations for gse_kernels.cu.
#pragma once

#include <cuda_runtime.h>

#include "gse_internal.cuh"

namespace gse {

// Green's-function geometry (CpuGreensFuncGSE.cpp:14-28), FP64 constants.
struct GreenGeom {
  int nfft[3];
  int half[3];   // nfft/2 + nfft%2: first index mapped to negative k
  int sizeX;     // nfft[0]/2 + 1 complex bins along x
  int nx_even;
  int want_energy;
  double twopi_box[3];
  double fourpi_vol;  // 4 pi / (nx ny nz): the c2r normalisation folded in
  double sigmafac;    // sigma^2 / 2
};

template <typename CT>
cudaError_t launch_spread(const typename Vec4<CT>::type* xyzq, int n, const Stencil<CT>& s,
                          CT* grid, long long* fixed_grid, cudaStream_t st);

template <typename CT>
cudaError_t launch_green_energy(typename Cplx<CT>::type* rhok, const GreenGeom& g,
                                double* partials, int np, double factor, double* energy_out,
                                cudaStream_t st);

template <typename CT>
cudaError_t launch_green_table(const GreenGeom& g, CT* tab, cudaStream_t st);

template <typename CT>
cudaError_t launch_green_apply(typename Cplx<CT>::type* rhok, const CT* tab, const GreenGeom& g,
                               double* partials, int np, double factor, double* energy_out,
                               cudaStream_t st);

// Reciprocal-space virial (xx, yy, zz, xy, xz, yz) of the half spectrum
// rhok with the Green's table tab; partials holds 6 * nblocks doubles, done is
// their zeroed counter (reset by the last block).
template <typename CT>
cudaError_t launch_virial(const typename Cplx<CT>::type* rhok, const CT* tab, const GreenGeom& g,
                          double half_sigma2, double factor, double* partials, unsigned* done,
                          int nblocks, double* out, cudaStream_t st);

// out[i] = in[i] with the charge set to 1 (in place allowed).
template <typename CT>
cudaError_t launch_unit_charges(const typename Vec4<CT>::type* in, typename Vec4<CT>::type* out,
                                int n, cudaStream_t st);

template <typename CT>
cudaError_t launch_dot_energy(const CT* a, const CT* b, long long size, double* partials, int np,
                              double factor, double* energy_out, cudaStream_t st);

template <typename CT>
cudaError_t launch_gather(const typename Vec4<CT>::type* xyzq, const int* perm, int n,
                          const Stencil<CT>& s, const CT* phi, double outscale, double* fx,
                          double* fy, double* fz, cudaStream_t st);

}  // namespace gse
