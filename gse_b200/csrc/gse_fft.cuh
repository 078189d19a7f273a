// gse_fft.cuh -- the mixed form's own 3-D real FFT solve for cubic grids of
// M = 16 * N2 points per side (N2 = 4 .. 12): launchers and the twiddle
// tables they read (gse_fft.cu).
#pragma once

#include <cuda_runtime.h>

#include "gse_internal.cuh"

namespace gse {

constexpr int kFftMinN2 = 4, kFftMaxN2 = 12;

// True when the grid is cubic with M = 16 * N2, N2 in [kFftMinN2, kFftMaxN2].
bool own_fft_supported(const int M[3]);

// Twiddle tables of one size in device memory, float2[16 N2 + 16 + N2]:
// w_M^(n1 k2) for n1 < 16, k2 < N2, then w_16^m, then w_N2^m, with
// w_N = exp(-2 pi i / N), each formed in double and rounded to float.
cudaError_t make_fft_twiddles(int M, float2** out);

// pdl (each launcher): the launch directly follows a kernel of this library
// on `st` and may overlap its end (programmatic dependent launch).
//
// Forward half, one CTA per z plane: the real x transform of two rows at a
// time and the y transform, rho -> rho^[z][y][x'] (x' <= M/2, FFTW's r2c
// layout and sign, unnormalised).  The input is the int64 fixed-point grid
// (g64 != nullptr, times `unscale`) or the float grid rho.  From the int64
// grid, rho_out (if not null) receives the float grid exactly as
// k_grid64_to_real writes it.  Where the plane fits in shared memory it is
// staged there by bulk copies; a copy wait that gives up sets kFlagStall in
// `flags` (may be NULL: not reported).  stall_test: the staged pass expects
// 16 bytes more than its first copy brings and waits about a millisecond, so
// that its first wait runs out (a test of that report; every copy completes).
cudaError_t launch_own_fft_xy_forward(int M, const long long* g64, const float* rho,
                                      double unscale, float* rho_out, float2* rhok,
                                      const float2* tw, int* flags, bool pdl, bool stall_test,
                                      cudaStream_t st);

// In place on rho^: the z transform of every (y, x') column, the multiply by
// the Green's table `tab` (same layout) with the k-space energy
// factor * sum_k w_k G |rho^|^2 into energy_out (w_k = 1 on the x' = 0 and
// x' = M/2 planes, 2 elsewhere; partials: the energy partials, done: their
// zeroed counter), and the inverse z transform.
cudaError_t launch_own_fft_z_green(int M, float2* rhok, const float* tab, const float2* tw,
                                   double* partials, unsigned* done, double factor,
                                   double* energy_out, bool pdl, cudaStream_t st);

// Inverse half, one CTA per z plane: the inverse y transform and the c2r x
// transform of two rows at a time (the imaginary parts of the x' = 0 and
// x' = M/2 bins are ignored, as FFTW's c2r does), unnormalised: rho^ -> phi.
// The half spectrum plane is staged by one bulk copy (flags as above).
cudaError_t launch_own_fft_xy_inverse(int M, const float2* rhok, float* phi, const float2* tw,
                                      int* flags, bool pdl, cudaStream_t st);

}  // namespace gse
