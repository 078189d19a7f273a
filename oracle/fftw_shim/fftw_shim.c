/*
 * fftw_shim.c -- FFTW-API entry points for the oracle's reference build.
 * Test infrastructure; see fftw3.h.  Array dimensions follow FFTW's
 * row-major convention: n0 is the slowest axis (z), n2 the fastest (x).
 */
#include <stdlib.h>
#include "fftw3.h"

int orc_fft_r2c_3d(int nx, int ny, int nz, const double* in, double* out);
int orc_fft_c2r_3d(int nx, int ny, int nz, const double* in, double* out);

struct orc_fftw_plan_s {
  int kind; /* 0 = r2c, 1 = c2r */
  int n0, n1, n2;
  void* in;
  void* out;
};

static fftw_plan make_plan(int kind, int n0, int n1, int n2, void* in, void* out) {
  fftw_plan p = (fftw_plan)malloc(sizeof(struct orc_fftw_plan_s));
  if (!p) return NULL;
  p->kind = kind;
  p->n0 = n0;
  p->n1 = n1;
  p->n2 = n2;
  p->in = in;
  p->out = out;
  return p;
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out,
                               unsigned flags) {
  (void)flags;
  return make_plan(0, n0, n1, n2, in, out);
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out,
                               unsigned flags) {
  (void)flags;
  return make_plan(1, n0, n1, n2, in, out);
}

void fftw_execute(const fftw_plan p) {
  if (!p) return;
  if (p->kind == 0)
    orc_fft_r2c_3d(p->n2, p->n1, p->n0, (const double*)p->in, (double*)p->out);
  else
    orc_fft_c2r_3d(p->n2, p->n1, p->n0, (const double*)p->in, (double*)p->out);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
