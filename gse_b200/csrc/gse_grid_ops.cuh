// gse_grid_ops.cuh -- launchers of the grid-to-grid operations of
// CpuGaussCharge beside the force path (gse_grid_ops.cu).
#pragma once

#include <cuda_runtime.h>

#include "gse_internal.cuh"

namespace gse {

// Taps of one axis of the on-grid convolution, G[i + n] for i = -n..n
// (CpuGaussCharge.cpp:428-438), built on the host in the reference's own
// expression and types.
template <typename CT>
struct ConvTaps {
  int n;
  CT g[kMaxStencil];
};

// One periodic 1-D pass along `axis` (0 = x, 1 = y, 2 = z):
// out[p] = sum_{i=-n..n} G[i + n] in[p + i e_axis], summed from zero in tap
// order with every product and sum rounded in CT.  in and out must not alias.
template <typename CT>
cudaError_t launch_conv_pass(const CT* in, CT* out, const int M[3], int axis,
                             const ConvTaps<CT>& taps, cudaStream_t st);

// Forward-difference field E_d = -(phi(p + e_d) - phi(p)) * inv_h[d]
// (CpuGaussCharge.cpp:62-98), periodic.
template <typename CT>
cudaError_t launch_efield(const CT* phi, CT* ex, CT* ey, CT* ez, const int M[3],
                          const CT inv_h[3], cudaStream_t st);

// Dipole sum of a charge grid (CpuGaussCharge.cpp:188-226): out[0..2] =
// sum_p (double)((rho_p hx hy hz) * (h_d i_d)).  partials holds 3 * kDipoleBlocks
// doubles; done is a zeroed counter that the last block resets.
constexpr int kDipoleBlocks = 592;  // capacity; launches use up to 4 per SM
template <typename CT>
cudaError_t launch_dipole(const CT* rho, const int M[3], const CT h[3], double* partials,
                          unsigned* done, double* out, cudaStream_t st);

}  // namespace gse
