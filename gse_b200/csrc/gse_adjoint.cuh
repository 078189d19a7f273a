// gse_adjoint.cuh -- launchers of the reverse-mode kernels (gse_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include "gse_internal.cuh"
#include "gse_tiled.cuh"

namespace gse {

cudaError_t launch_batch_adj_source(const float4* xyzq, const int* perm, int ntot,
                                    const BatchSys* sys, const int* first, int nsys, double c,
                                    const double* gfx, const double* gfy, const double* gfz,
                                    float* lambda, cudaStream_t st);
cudaError_t launch_batch_adj_gather(const float4* xyzq, const int* perm, int ntot,
                                    const BatchSys* sys, const int* first, int nsys, double c,
                                    const double* dLdE, const float* psi, const float* phi,
                                    const double* gfx, const double* gfy, const double* gfz,
                                    double* dq, double* dx, double* dy, double* dz,
                                    cudaStream_t st);

// Tiled reverse pass of the mixed form (sorted atoms and bin starts as the
// forward pass leaves them).  The source lambda is accumulated in `grid64`
// (cleared here) and written as floats into `lambda`.
cudaError_t launch_adj_scatter(const float4* sorted, const int* perm, const int* start,
                               const BinLayout& b, const Stencil<float>& sg, double c,
                               const double* gfx, const double* gfy, const double* gfz,
                               long long* grid64, float* lambda, cudaStream_t st);
cudaError_t launch_adj_gather_tiled(const float4* sorted, const int* perm, const int* start,
                                    const BinLayout& b, const Stencil<float>& sp,
                                    const Stencil<float>& sg, double c, double gE_ch3,
                                    const float* psi, const float* phi, const double* gfx,
                                    const double* gfy, const double* gfz, double* dq, double* dx,
                                    double* dy, double* dz, cudaStream_t st);
cudaError_t launch_batch_adj_scatter(const float4* sorted, const int* perm, const int* start,
                                     const BatchSys* sys, const BatchItem* items,
                                     const BatchSeg* segs, int nseg, int ctas, double c,
                                     const double* gfx, const double* gfy, const double* gfz,
                                     long long* grid64, long long gsize, float* lambda,
                                     cudaStream_t st);
cudaError_t launch_batch_adj_gather_tiled(const float4* sorted, const int* perm, const int* start,
                                          const BatchSys* sys, const BatchItem* items,
                                          const BatchSeg* segs, int nseg, int ctas, double c,
                                          const double* dLdE, const float* psi, const float* phi,
                                          const double* gfx, const double* gfy, const double* gfz,
                                          double* dq, double* dx, double* dy, double* dz,
                                          cudaStream_t st);

template <typename CT>
cudaError_t launch_adj_source(const typename Vec4<CT>::type* xyzq, const int* perm, int n,
                              const Stencil<CT>& s, double c, const double* gfx,
                              const double* gfy, const double* gfz, CT* lambda, cudaStream_t st);

template <typename CT>
cudaError_t launch_adj_gather(const typename Vec4<CT>::type* xyzq, const int* perm, int n,
                              const Stencil<CT>& sp, const Stencil<CT>& sg, double c,
                              double gE_ch3, const CT* psi, const CT* phi, const double* gfx,
                              const double* gfy, const double* gfz, double* dq, double* dx,
                              double* dy, double* dz, cudaStream_t st);

}  // namespace gse
