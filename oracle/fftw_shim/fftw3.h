/*
 * fftw3.h -- FFTW-API shim used ONLY to compile the reference's CpuFFTSolver
 * (CpuFFTSolver.cpp:19-23,41-44,61-64,88,94 of ap-hynninen/GSE) into the
 * oracle's reference build (oracle/_ref).  FFTW itself is absent from this
 * image; the six entry points below are backed by the project-written FFT in
 * oracle/gse_oracle.c, pinned against numpy.fft by the tests.
 * Test infrastructure; not part of the product library.
 */
#ifndef GSE_ORACLE_FFTW3_SHIM_H
#define GSE_ORACLE_FFTW3_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct orc_fftw_plan_s* fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out,
                               unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif
#endif
