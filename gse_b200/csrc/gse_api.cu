// gse_api.cu -- C ABI of the GSE-k library (include/gse_b200.h).
//
// One gse_context owns, on one device and one stream: the rhoS and phiM grids
// (CpuGSE.h:38-42), the k-space buffer rhoK (CpuFFTSolver.h:24), the int64
// fixed-point accumulation grid of the mixed form, cuFFT plans (replacing
// the FFTW plans of CpuFFTSolver.cpp:28-69), and staging buffers for atoms
// and forces.
#include <cufft.h>
#include <cufftXt.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "gse_b200.h"
#include "gse_internal.cuh"
#include "gse_kernels.cuh"
#include "gse_adjoint.cuh"
#include "gse_ewald.cuh"
#include "gse_fft.cuh"
#include "gse_grid_ops.cuh"
#include "gse_tiled.cuh"
#include "gse_green_cb_fatbin.h"  // generated: the c2r load callbacks as LTO code

using namespace gse;

namespace {

thread_local std::string g_last_error;

gse_status_t fail(gse_status_t s, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
gse_status_t fail(gse_status_t s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

#define CU(call)                                                                            \
  do {                                                                                      \
    cudaError_t _e = (call);                                                                \
    if (_e != cudaSuccess)                                                                  \
      return fail(_e == cudaErrorMemoryAllocation ? GSE_ERR_OOM : GSE_ERR_CUDA,             \
                  "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e));       \
  } while (0)

#define CUFFT(call)                                                                         \
  do {                                                                                      \
    cufftResult _r = (call);                                                                \
    if (_r != CUFFT_SUCCESS)                                                                \
      return fail(_r == CUFFT_ALLOC_FAILED ? GSE_ERR_OOM : GSE_ERR_CUDA,                    \
                  "%s:%d %s: cufft error %d", __FILE__, __LINE__, #call, (int)_r);          \
  } while (0)

#define TRY(call)                                                                           \
  do {                                                                                      \
    gse_status_t _s = (call);                                                               \
    if (_s != GSE_OK) return _s;                                                            \
  } while (0)

// capacity of the reductions' per-block partial sums (+1 counter slot); the
// reductions launch at most this many blocks
constexpr int kEnergyPartials = 2368;

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Page-locked host memory (cudaHostAlloc / cudaHostRegister): copies to and
// from it can be recorded in a CUDA graph.
bool is_pinned_host(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

}  // namespace

namespace gse {
gse_status_t set_error(gse_status_t s, const char* msg) { return fail(s, "%s", msg); }

// A caller's pointer that a kernel may read or write in place.  NULL and host
// memory pass: host memory only reaches the GPU through cudaMemcpyAsync into
// the library's own buffers.  Device memory must belong to `device` (a kernel
// of this context cannot address another GPU's allocation) and start on an
// `align`-byte boundary: the kernels read position records as float4/double4,
// forces and gradients as doubles and spectra as float4/double2 vectors, and a
// misaligned vector access faults.  The check runs on the host, before any
// work of the call is queued.
gse_status_t check_ptr(const void* p, int device, size_t align, const char* what) {
  if (!p) return GSE_OK;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return GSE_OK;
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) return GSE_OK;
  if (a.type == cudaMemoryTypeDevice && a.device != device)
    return fail(GSE_ERR_INVALID_ARG, "%s is memory of device %d, the call runs on device %d", what,
                a.device, device);
  if (align > 1 && (uintptr_t)p % align != 0)
    return fail(GSE_ERR_INVALID_ARG, "%s is device memory that is not %zu-byte aligned", what,
                align);
  return GSE_OK;
}
}  // namespace gse

namespace {
using gse::check_ptr;

// The three per-atom double arrays of a force, field or gradient output.
gse_status_t check_xyz(int device, const double* x, const double* y, const double* z,
                       const char* what) {
  TRY(check_ptr(x, device, sizeof(double), what));
  TRY(check_ptr(y, device, sizeof(double), what));
  TRY(check_ptr(z, device, sizeof(double), what));
  return GSE_OK;
}
}  // namespace

struct gse_context {
  gse_params_t p;
  cudaStream_t stream = nullptr;
  bool fp64 = true;
  size_t ct = 8;  // sizeof(CT)
  double sigma1 = 0, sigma2 = 0, rcut1 = 0;
  long long size = 0;   // real grid points
  long long ksize = 0;  // complex half-spectrum bins
  void* d_rho = nullptr;
  void* d_phi = nullptr;
  void* d_rhok = nullptr;
  long long* d_fixed = nullptr;
  void* d_xyzq = nullptr;
  void* d_sorted = nullptr;
  int* d_perm = nullptr;
  size_t atom_cap = 0;
  // binning of the tiled kernels (stable sort by z cell, y cell, x bin)
  BinLayout bl{};
  int nbins2 = 0;
  int* d_bkey = nullptr;
  int* d_btmp = nullptr;
  int* d_bcounts = nullptr;
  int* d_bstart = nullptr;
  int* d_blstart = nullptr;  // mixed form: tile-local bin starts of the scan
  int* d_btiles = nullptr;
  unsigned* d_qmax = nullptr;
  // Green's function table of the context's own solve (sigma2, box)
  void* d_gtab = nullptr;
  bool gtab_valid = false;
  // adjoint staging: upstream force gradients (3 x cap) and outputs (4 x cap)
  double* d_adj = nullptr;
  size_t adj_cap = 0;
  double* d_force = nullptr;  // 3 x atom_cap
  double* d_partials = nullptr;
  double* d_scalars = nullptr;  // [0] energy of the last solve, [1] scratch, [4..6] dipole,
                                // [8..13] virial
  // grid scratch of the stand-alone grid operations, allocated on first use
  void* d_scratch = nullptr;
  size_t scratch_bytes = 0;
  int* d_bad = nullptr;
  double* h_pinned = nullptr;  // [0] energy
  // set by the binning when a position or charge is not finite; host memory
  // mapped into the device, so reading it after a synchronisation costs no copy
  volatile int* h_bad = nullptr;
  int* d_badmap = nullptr;
  cufftHandle plan_f = 0, plan_b = 0;
  bool plans = false;
  // c2r plan whose load callback multiplies by the Green's table (the solve
  // of the context's own sigma2 and box; plan_b stays plain for the others)
  cufftHandle plan_bg = 0;
  bool green_cb = false;     // plan_bg exists and is used
  bool green_cb_tried = false;
  // the mixed form's own 3-D FFT solve (cubic M = 16 N2): its twiddles, and
  // whether the float rho grid still has to be made from the int64 grid
  float2* d_fft_tw = nullptr;
  bool own_fft = false;
  // GSE_B200_TEST_FFT_STALL=1 at creation: the staged forward plane pass's
  // first copy wait runs out (about a millisecond), a test of the
  // GSE_ERR_TIMEOUT report
  bool fft_stall_test = false;
  bool fixed_pending = false;
  bool rho_valid = false, phi_valid = false, energy_valid = false;
  // replay of repeated gse_forward calls with device inputs and outputs: the
  // second identical call is captured into a CUDA graph, later ones launch it
  struct FwdKey {
    int n = -1;
    const void* x = nullptr;
    double *e = nullptr, *fx = nullptr, *fy = nullptr, *fz = nullptr;
    double box[3] = {0, 0, 0};
    cudaStream_t stream = nullptr;
    bool operator==(const FwdKey& o) const {
      return n == o.n && x == o.x && e == o.e && fx == o.fx && fy == o.fy && fz == o.fz &&
             box[0] == o.box[0] && box[1] == o.box[1] && box[2] == o.box[2] &&
             stream == o.stream;
    }
  } fwd_key;
  cudaGraphExec_t fwd_exec = nullptr;
  long long fwd_launches = 0;
  bool fwd_graphs = true;
  // classification of the pointers of the captured call, for the replay path
  bool fwd_host_io = false, fwd_e_host = false;
  const double* fwd_e_raw = nullptr;
  // optional per-stage device timing (gse_set_timing)
  bool timing = false;
  cudaEvent_t ev[GSE_NUM_STAGES][2] = {};
  bool ev_pending[GSE_NUM_STAGES] = {};
  double stage_ms[GSE_NUM_STAGES] = {};
  long long stage_count[GSE_NUM_STAGES] = {};
  long long launches = 0;  // kernels of this library launched so far
};

namespace {

// Fold a completed start/stop pair into the stage totals.
void harvest(gse_context_t* c, int st) {
  if (!c->ev_pending[st]) return;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, c->ev[st][0], c->ev[st][1]) == cudaSuccess) {
    c->stage_ms[st] += ms;
    c->stage_count[st] += 1;
  } else {
    cudaGetLastError();
  }
  c->ev_pending[st] = false;
}

// RAII bracket of one stage on the context stream.
struct StageTimer {
  gse_context_t* c;
  int st;
  StageTimer(gse_context_t* c_, int st_) : c(c_), st(st_) {
    if (!c->timing) return;
    if (c->ev_pending[st]) {
      cudaEventSynchronize(c->ev[st][1]);
      harvest(c, st);
    }
    cudaEventRecord(c->ev[st][0], c->stream);
  }
  ~StageTimer() {
    if (!c->timing) return;
    cudaEventRecord(c->ev[st][1], c->stream);
    c->ev_pending[st] = true;
  }
};

gse_status_t check_ctx(gse_context_t* c) {
  if (!c) return fail(GSE_ERR_INVALID_ARG, "NULL context");
  cudaError_t e = cudaSetDevice(c->p.device);
  if (e != cudaSuccess) return fail(GSE_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  return GSE_OK;
}

template <typename CT>
Stencil<CT> stencil_of(const gse_context_t* c, const double box[3], double sigma, double rcut,
                       bool gather, bool normalize) {
  const int M[3] = {c->p.size_x, c->p.size_y, c->p.size_z};
  Stencil<CT> s = make_stencil<CT>(M, box, sigma, rcut, gather, normalize, 1.0);
  s.fixed_scale = fixed_scale_for((double)make_stencil<CT>(M, box, sigma, rcut, false, false, 1.0).pref);
  return s;
}

struct Box3 {
  double v[3];
};
Box3 ctx_box(const gse_context_t* c) { return Box3{{c->p.box_x, c->p.box_y, c->p.box_z}}; }

gse_status_t check_stencil(const gse_context_t* c, const double box[3], double sigma,
                           double rcut) {
  if (!(sigma > 0.0) || !(rcut > 0.0) || !std::isfinite(sigma) || !std::isfinite(rcut))
    return fail(GSE_ERR_INVALID_ARG, "sigma and rcut must be positive and finite");
  for (int d = 0; d < 3; d++)
    if (!(box[d] > 0.0) || !std::isfinite(box[d]))
      return fail(GSE_ERR_INVALID_ARG, "box lengths must be positive and finite");
  const int M[3] = {c->p.size_x, c->p.size_y, c->p.size_z};
  for (int d = 0; d < 3; d++) {
    const int n = (int)std::ceil(rcut / (box[d] / (double)M[d]));
    if (2 * n + 1 > kMaxStencil)
      return fail(GSE_ERR_STENCIL_TOO_LARGE, "stencil 2n+1=%d exceeds %d on axis %d", 2 * n + 1,
                  kMaxStencil, d);
  }
  return GSE_OK;
}

// Forget the captured forward graph (its buffers or parameters change).
void drop_fwd_graph(gse_context_t* c) {
  if (c->fwd_exec) cudaGraphExecDestroy(c->fwd_exec);
  c->fwd_exec = nullptr;
  c->fwd_key = gse_context_t::FwdKey();
}

gse_status_t ensure_atoms(gse_context_t* c, int n) {
  if ((size_t)n <= c->atom_cap) return GSE_OK;
  drop_fwd_graph(c);
  size_t cap = c->atom_cap ? c->atom_cap : 1024;
  while (cap < (size_t)n) cap *= 2;
  cudaFree(c->d_xyzq);
  cudaFree(c->d_sorted);
  cudaFree(c->d_perm);
  cudaFree(c->d_force);
  cudaFree(c->d_bkey);
  cudaFree(c->d_btmp);
  c->d_xyzq = c->d_sorted = nullptr;
  c->d_perm = nullptr;
  c->d_force = nullptr;
  c->d_bkey = c->d_btmp = nullptr;
  c->atom_cap = 0;
  const size_t rec = 4 * c->ct;
  CU(cudaMalloc(&c->d_xyzq, cap * rec));
  CU(cudaMalloc(&c->d_sorted, cap * rec));
  CU(cudaMalloc(&c->d_perm, cap * sizeof(int)));
  CU(cudaMalloc(&c->d_force, 3 * cap * sizeof(double)));
  CU(cudaMalloc(&c->d_bkey, cap * sizeof(int)));
  CU(cudaMalloc(&c->d_btmp, cap * sizeof(int)));
  c->atom_cap = cap;
  return GSE_OK;
}

// Returns a device pointer to the n records (copied in if host memory).
gse_status_t stage_atoms(gse_context_t* c, int n, const void* xyzq, const void** dptr) {
  if (n < 0) return fail(GSE_ERR_INVALID_ARG, "negative atom count");
  if (n > 0 && !xyzq) return fail(GSE_ERR_INVALID_ARG, "NULL xyzq");
  TRY(check_ptr(xyzq, c->p.device, 4 * c->ct, "xyzq"));
  TRY(ensure_atoms(c, n > 0 ? n : 1));
  if (n == 0) {
    *dptr = c->d_xyzq;
    return GSE_OK;
  }
  if (is_device_ptr(xyzq)) {
    *dptr = xyzq;
  } else {
    CU(cudaMemcpyAsync(c->d_xyzq, xyzq, (size_t)n * 4 * c->ct, cudaMemcpyHostToDevice,
                       c->stream));
    *dptr = c->d_xyzq;
  }
  return GSE_OK;
}

// Stable counting sort of the atoms into c->d_sorted / c->d_perm by
// (z cell, y cell, x bin) of their stencil centres; c->d_bstart holds the bin
// offsets afterwards.
// clear_fixed: the counting kernel also clears the mixed form's int64 grid.
template <typename CT>
gse_status_t bin_atoms(gse_context_t* c, int n, const void* dx, const Stencil<CT>& s,
                       bool clear_fixed = false) {
  typedef typename Vec4<CT>::type V;
  StageTimer tm(c, GSE_STAGE_BIN);
  BinScratch w{c->d_bkey, c->d_bcounts, c->d_bstart, c->d_btiles, c->d_btmp, c->d_qmax,
               c->d_badmap};
  // mixed: count, a tile-local scan and the placement that applies the tile
  // offsets (the counts stay zero between calls); FP64: count, three scan
  // passes and a stable placement in two kernels
  if (!c->fp64) {
    w.lstart = c->d_blstart;
    w.counts_zero = true;
    if (clear_fixed) {
      w.clear = c->d_fixed;
      w.clear_n = c->size;
    }
  }
  c->launches += c->fp64 ? (n > 0 ? 6 : 3) : (n > 0 ? 3 : 2);
  CU(launch_bin_sorted<CT>((const V*)dx, n, c->bl, s.inv_h[0], s.inv_h[1], s.inv_h[2], w,
                           (V*)c->d_sorted, c->d_perm, c->stream));
  return GSE_OK;
}

// Size the scatter buffers for stencil width W (once per width).
template <typename CT>
bool tiled_ok(const gse_context_t* c, const Stencil<CT>& s) {
  return spread_tiled_supported<CT>(s) && c->p.size_x >= kMinTiledGrid &&
         c->p.size_y >= kMinTiledGrid && c->p.size_z >= kMinTiledGrid;
}

// Spread into c->d_rho.  `presorted`: c->d_sorted / d_bstart already hold the
// binned atoms of this call.
template <typename CT>
// `defer_rho`: with the own FFT, leave the float grid to the solve that
// follows (it reads the int64 grid directly and writes rho on the way).
// `zeroed`: the int64 grid was cleared before the binning that directly
// precedes this call (forward_body).
gse_status_t do_spread(gse_context_t* c, int n, const void* dx, const double box[3], double sigma,
                       double rcut, bool normalize, bool presorted = false,
                       bool defer_rho = false, bool zeroed = false) {
  typedef typename Vec4<CT>::type V;
  const Stencil<CT> s = stencil_of<CT>(c, box, sigma, rcut, false, normalize);
  if (!normalize && tiled_ok<CT>(c, s)) {
    if (!presorted) TRY(bin_atoms<CT>(c, n, dx, s));
    StageTimer tm(c, GSE_STAGE_SPREAD);
    if (c->fp64) {
      c->launches += 1;
      CU(launch_spread_tiled<CT>((const V*)c->d_sorted, c->d_bstart, c->d_qmax, c->bl, s,
                                 (CT*)c->d_rho, c->stream));
    } else if constexpr (sizeof(CT) == 4) {
      const bool defer = defer_rho && c->own_fft;
      c->launches += defer ? 1 : 2;
      CU(launch_spread_scatter((const float4*)c->d_sorted, c->d_bstart, c->bl, s, c->d_fixed,
                               defer ? nullptr : (float*)c->d_rho, zeroed && presorted,
                               c->stream));
      c->fixed_pending = defer;
    }
  } else {
    StageTimer tm(c, GSE_STAGE_SPREAD);
    c->launches += (n > 0 ? 1 : 0) + (c->fp64 ? 0 : 1);
    CU(launch_spread<CT>((const V*)dx, n, s, (CT*)c->d_rho, c->fp64 ? nullptr : c->d_fixed,
                         c->stream));
  }
  c->rho_valid = true;
  c->phi_valid = false;
  c->energy_valid = false;
  return GSE_OK;
}

// after_solve: the gather directly follows the own FFT's last kernel on the
// stream (forward_body), so it may be launched as that kernel's dependent.
template <typename CT>
gse_status_t do_gather(gse_context_t* c, int n, const void* dx, const double box[3], double sigma,
                       double rcut, const CT* phi, double outscale, double* fx, double* fy,
                       double* fz, bool presorted = false, bool after_solve = false) {
  typedef typename Vec4<CT>::type V;
  const Stencil<CT> s = stencil_of<CT>(c, box, sigma, rcut, true, false);
  if (n == 0) return GSE_OK;
  if (!presorted) TRY(bin_atoms<CT>(c, n, dx, s));
  StageTimer tm(c, GSE_STAGE_GATHER);
  c->launches += 1;
  if (tiled_ok<CT>(c, s))
    CU(launch_gather_tiled<CT>((const V*)c->d_sorted, c->d_perm, c->d_bstart, c->bl, s, phi,
                               outscale, fx, fy, fz,
                               after_solve && presorted && c->own_fft && !c->timing, c->stream));
  else
    CU(launch_gather<CT>((const V*)c->d_sorted, c->d_perm, n, s, phi, outscale, fx, fy, fz,
                         c->stream));
  return GSE_OK;
}

GreenGeom green_geom(const gse_context_t* c, double sigma, double bx, double by, double bz,
                     bool energy) {
  GreenGeom g;
  g.nfft[0] = c->p.size_x;
  g.nfft[1] = c->p.size_y;
  g.nfft[2] = c->p.size_z;
  for (int d = 0; d < 3; d++) g.half[d] = g.nfft[d] / 2 + (g.nfft[d] % 2);
  g.sizeX = g.nfft[0] / 2 + 1;
  g.nx_even = (g.nfft[0] % 2) == 0;
  g.want_energy = energy ? 1 : 0;
  g.twopi_box[0] = 2.0 * kPi / bx;
  g.twopi_box[1] = 2.0 * kPi / by;
  g.twopi_box[2] = 2.0 * kPi / bz;
  g.fourpi_vol = 4.0 * kPi / (double)(g.nfft[0] * g.nfft[1] * g.nfft[2]);
  g.sigmafac = sigma * sigma / 2.0;
  return g;
}

double energy_factor(const gse_context_t* c) {
  // CpuGSE.cpp:99-102: energy *= ccelec*hx*hy*hz*0.5
  const double hx = c->p.box_x / (double)c->p.size_x;
  const double hy = c->p.box_y / (double)c->p.size_y;
  const double hz = c->p.box_z / (double)c->p.size_z;
  return c->p.ccelec * hx * hy * hz * 0.5;
}

gse_status_t fft_forward(gse_context_t* c, const void* rho, void* rhok) {
  if (c->fp64)
    CUFFT(cufftExecD2Z(c->plan_f, (cufftDoubleReal*)rho, (cufftDoubleComplex*)rhok));
  else
    CUFFT(cufftExecR2C(c->plan_f, (cufftReal*)rho, (cufftComplex*)rhok));
  return GSE_OK;
}

gse_status_t fft_backward(gse_context_t* c, void* rhok, void* phi) {
  if (c->fp64)
    CUFFT(cufftExecZ2D(c->plan_b, (cufftDoubleComplex*)rhok, (cufftDoubleReal*)phi));
  else
    CUFFT(cufftExecC2R(c->plan_b, (cufftComplex*)rhok, (cufftReal*)phi));
  return GSE_OK;
}

// phi = c2r(G(sigma) r2c(rho)); optionally the k-space energy into d_scalars[0].
gse_status_t do_solve(gse_context_t* c, const void* rho, void* phi, double sigma, double bx,
                      double by, double bz, bool energy) {
  {
    StageTimer tm(c, GSE_STAGE_FFT_FORWARD);
    TRY(fft_forward(c, rho, c->d_rhok));
  }
  {
    StageTimer tm(c, GSE_STAGE_GREEN);
    const GreenGeom g = green_geom(c, sigma, bx, by, bz, energy);
    c->launches += energy ? 2 : 1;
    if (c->fp64)
      CU(launch_green_energy<double>((double2*)c->d_rhok, g, c->d_partials, kEnergyPartials,
                                     energy_factor(c), c->d_scalars, c->stream));
    else
      CU(launch_green_energy<float>((float2*)c->d_rhok, g, c->d_partials, kEnergyPartials,
                                    energy_factor(c), c->d_scalars, c->stream));
  }
  StageTimer tm(c, GSE_STAGE_FFT_BACKWARD);
  TRY(fft_backward(c, c->d_rhok, phi));
  return GSE_OK;
}

// The context's own solve (sigma2, context box) with the tabulated Green's
// function: r2c -> multiply + energy -> c2r.
// Grids from this size on use the callback plan: its cuFFT link step takes
// about half a second once per context, which smaller grids do not earn back.
constexpr long long kGreenCallbackMinPoints = 64LL * 64 * 64;

// The context's c2r plan with the Green multiply as a load callback (cuFFT's
// link-time callbacks).  false: the callback plan is not available here and
// the solve keeps its separate multiply kernel.
bool make_green_callback_plan(gse_context_t* c) {
  cufftHandle pl = 0;
  if (cufftCreate(&pl) != CUFFT_SUCCESS) return false;
  const char* sym = c->fp64 ? "gse_green_load_z" : "gse_green_load_c";
  size_t ws = 0;
  const bool ok =
      cufftXtSetJITCallback(pl, sym, gse_green_cb_fatbin, sizeof(gse_green_cb_fatbin),
                            c->fp64 ? CUFFT_CB_LD_COMPLEX_DOUBLE : CUFFT_CB_LD_COMPLEX,
                            &c->d_gtab) == CUFFT_SUCCESS &&
      cufftMakePlan3d(pl, c->p.size_z, c->p.size_y, c->p.size_x,
                      c->fp64 ? CUFFT_Z2D : CUFFT_C2R, &ws) == CUFFT_SUCCESS &&
      cufftSetStream(pl, c->stream) == CUFFT_SUCCESS;
  if (!ok) {
    cufftDestroy(pl);
    cudaGetLastError();
    return false;
  }
  c->plan_bg = pl;
  return true;
}

gse_status_t do_solve_ctx(gse_context_t* c) {
  const GreenGeom g = green_geom(c, c->sigma2, c->p.box_x, c->p.box_y, c->p.box_z, true);
  if (!c->d_gtab) CU(cudaMalloc(&c->d_gtab, c->ksize * c->ct));  // fixed address from here on
  if (c->own_fft) {
    // mixed form, cubic M = 16 N2: three passes of this library's own FFT;
    // the Green's multiply and the k-space energy sit in the z pass
    if (!c->gtab_valid) {
      CU(launch_green_table<float>(g, (float*)c->d_gtab, c->stream));
      c->gtab_valid = true;
    }
    const int M = c->p.size_x;
    {
      StageTimer tm(c, GSE_STAGE_FFT_FORWARD);
      c->launches += 1;
      const bool fx = c->fixed_pending;
      // from a deferred spread (forward_body) the solve follows the spread
      // kernel directly, and each pass follows the previous one: dependent
      // launches, unless stage timing puts events between them
      CU(launch_own_fft_xy_forward(M, fx ? c->d_fixed : nullptr, fx ? nullptr : (float*)c->d_rho,
                                   std::exp2(-(double)kFlushBits), fx ? (float*)c->d_rho : nullptr,
                                   (float2*)c->d_rhok, c->d_fft_tw, c->bl.flags,
                                   fx && !c->timing, c->fft_stall_test, c->stream));
      c->fixed_pending = false;
    }
    {
      StageTimer tm(c, GSE_STAGE_GREEN);
      c->launches += 1;
      CU(launch_own_fft_z_green(M, (float2*)c->d_rhok, (const float*)c->d_gtab, c->d_fft_tw,
                                c->d_partials,
                                reinterpret_cast<unsigned*>(c->d_partials + kEnergyPartials),
                                energy_factor(c), c->d_scalars, !c->timing, c->stream));
    }
    StageTimer tm(c, GSE_STAGE_FFT_BACKWARD);
    c->launches += 1;
    CU(launch_own_fft_xy_inverse(M, (const float2*)c->d_rhok, (float*)c->d_phi, c->d_fft_tw,
                                 c->bl.flags, !c->timing, c->stream));
    return GSE_OK;
  }
  if (!c->green_cb_tried && c->size >= kGreenCallbackMinPoints) {
    // linked once, on the first solve outside any stream capture
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(c->stream, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
      c->green_cb = make_green_callback_plan(c);
      c->green_cb_tried = true;
    }
    cudaGetLastError();
  }
  if (!c->gtab_valid) {
    if (c->fp64)
      CU(launch_green_table<double>(g, (double*)c->d_gtab, c->stream));
    else
      CU(launch_green_table<float>(g, (float*)c->d_gtab, c->stream));
    c->gtab_valid = true;
  }
  {
    StageTimer tm(c, GSE_STAGE_FFT_FORWARD);
    TRY(fft_forward(c, c->d_rho, c->d_rhok));
  }
  if (c->green_cb) {
    // Green multiply inside the c2r (load callback); the energy then as the
    // reference computes it, 1/2 ccelec h^3 sum rho phi (CpuGSE.cpp:86-103)
    {
      StageTimer tm(c, GSE_STAGE_FFT_BACKWARD);
      if (c->fp64)
        CUFFT(cufftExecZ2D(c->plan_bg, (cufftDoubleComplex*)c->d_rhok, (cufftDoubleReal*)c->d_phi));
      else
        CUFFT(cufftExecC2R(c->plan_bg, (cufftComplex*)c->d_rhok, (cufftReal*)c->d_phi));
    }
    StageTimer tm(c, GSE_STAGE_GREEN);
    c->launches += 1;
    if (c->fp64)
      CU(launch_dot_energy<double>((const double*)c->d_rho, (const double*)c->d_phi, c->size,
                                   c->d_partials, kEnergyPartials, energy_factor(c),
                                   c->d_scalars, c->stream));
    else
      CU(launch_dot_energy<float>((const float*)c->d_rho, (const float*)c->d_phi, c->size,
                                  c->d_partials, kEnergyPartials, energy_factor(c),
                                  c->d_scalars, c->stream));
    return GSE_OK;
  }
  {
    StageTimer tm(c, GSE_STAGE_GREEN);
    c->launches += 1;
    if (c->fp64)
      CU(launch_green_apply<double>((double2*)c->d_rhok, (const double*)c->d_gtab, g,
                                    c->d_partials, kEnergyPartials, energy_factor(c),
                                    c->d_scalars, c->stream));
    else
      CU(launch_green_apply<float>((float2*)c->d_rhok, (const float*)c->d_gtab, g, c->d_partials,
                                   kEnergyPartials, energy_factor(c), c->d_scalars, c->stream));
  }
  StageTimer tm(c, GSE_STAGE_FFT_BACKWARD);
  TRY(fft_backward(c, c->d_rhok, c->d_phi));
  return GSE_OK;
}

// Copy `bytes` from device src to dst (host or device) on the stream.
gse_status_t copy_out(gse_context_t* c, void* dst, const void* src, size_t bytes, bool* host) {
  const bool dev = is_device_ptr(dst);
  CU(cudaMemcpyAsync(dst, src, bytes, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     c->stream));
  if (!dev) *host = true;
  return GSE_OK;
}

// After a synchronisation: report (once) non-finite inputs or a charge
// density beyond the mixed form's fixed-point range seen since the last
// report.
gse_status_t check_finite(gse_context_t* c) {
  if (c->h_bad && *c->h_bad) {
    const int f = *c->h_bad;
    *c->h_bad = 0;
    if (f == kFlagStall)
      return fail(GSE_ERR_TIMEOUT, "a bounded wait for a staged copy in the FFT gave up");
    if (f == kFlagRange)
      return fail(GSE_ERR_RANGE,
                  "the charge in one 16^3-cell brick exceeds the mixed form's fixed-point range "
                  "(sum of |q| (2 pi sigma1^2)^-1.5 over the brick above about 2^19, or one "
                  "charge's above 2^11); use the FP64 form");
    return fail(GSE_ERR_NONFINITE, "a position or charge is NaN or infinite");
  }
  return GSE_OK;
}

gse_status_t finish(gse_context_t* c, bool host_outputs) {
  if (host_outputs) {
    CU(cudaStreamSynchronize(c->stream));
    TRY(check_finite(c));
  }
  CU(cudaGetLastError());
  return GSE_OK;
}

// Gather into fx/fy/fz (host or device, any may be NULL).
template <typename CT>
gse_status_t gather_to(gse_context_t* c, int n, const void* dx, const double box[3], double sigma,
                       double rcut, const CT* phi, double outscale, double* fx, double* fy,
                       double* fz, bool* host, bool presorted = false, bool after_solve = false) {
  const bool direct = fx && fy && fz && is_device_ptr(fx) && is_device_ptr(fy) && is_device_ptr(fz);
  if (direct)
    return do_gather<CT>(c, n, dx, box, sigma, rcut, phi, outscale, fx, fy, fz, presorted,
                         after_solve);
  double* f = c->d_force;
  // three outputs that are consecutive rows of one [3][n] array take one copy
  const bool rows = fx && fy == fx + n && fz == fx + 2 * (size_t)n;
  const size_t stride = rows ? (size_t)n : c->atom_cap;
  TRY(do_gather<CT>(c, n, dx, box, sigma, rcut, phi, outscale, f, f + stride, f + 2 * stride,
                    presorted, after_solve));
  if (n == 0) return GSE_OK;
  if (rows) return copy_out(c, fx, f, 3 * (size_t)n * sizeof(double), host);
  if (fx) TRY(copy_out(c, fx, f, n * sizeof(double), host));
  if (fy) TRY(copy_out(c, fy, f + stride, n * sizeof(double), host));
  if (fz) TRY(copy_out(c, fz, f + 2 * stride, n * sizeof(double), host));
  return GSE_OK;
}

gse_status_t energy_out(gse_context_t* c, double* energy, bool* host) {
  if (!energy) return GSE_OK;
  if (is_device_ptr(energy)) {
    CU(cudaMemcpyAsync(energy, c->d_scalars, sizeof(double), cudaMemcpyDeviceToDevice,
                       c->stream));
  } else {
    CU(cudaMemcpyAsync(c->h_pinned, c->d_scalars, sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
    CU(cudaStreamSynchronize(c->stream));
    *energy = c->h_pinned[0];
    *host = true;
  }
  return GSE_OK;
}

}  // namespace

// Helpers of the grid operations beside the force path.
namespace {

// At least `bytes` of grid scratch on the context's device.
gse_status_t ensure_scratch(gse_context_t* c, size_t bytes) {
  if (c->scratch_bytes >= bytes) return GSE_OK;
  CU(cudaStreamSynchronize(c->stream));
  cudaFree(c->d_scratch);
  c->d_scratch = nullptr;
  c->scratch_bytes = 0;
  if (cudaMalloc(&c->d_scratch, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(GSE_ERR_OOM, "grid scratch of %zu bytes", bytes);
  }
  c->scratch_bytes = bytes;
  return GSE_OK;
}

// Taps of the on-grid convolution, CpuGaussCharge.cpp:413-438, in the
// reference's own expressions and types: the exponent is formed in CT and
// handed to the double exp() (the overload an unqualified exp() of a float
// resolves to there); the z taps multiply the CT prefactor by that double
// before rounding to CT.
template <typename CT>
void conv_taps(const int M[3], const double box[3], double sigma, double rcut,
               ConvTaps<CT> taps[3]) {
  double hd[3];
  for (int d = 0; d < 3; d++) hd[d] = box[d] / (double)M[d];
  const CT inv_2sigmasq = (CT)(1.0 / (2.0 * sigma * sigma));
  const CT pref = (CT)(std::pow(2.0 * kPi * sigma * sigma, -3.0 / 2.0) * hd[0] * hd[1] * hd[2]);
  for (int d = 0; d < 3; d++) {
    const int n = (int)std::ceil(rcut / hd[d]);
    const CT hsq = (CT)(hd[d] * hd[d]);
    taps[d].n = n;
    for (int i = -n; i <= n; i++) {
      const CT arg = -hsq * (CT)(i * i) * inv_2sigmasq;
      const double e = std::exp((double)arg);
      taps[d].g[i + n] = d == 2 ? (CT)((double)pref * e) : (CT)e;
    }
  }
}

template <typename CT>
gse_status_t spread_on_grid(gse_context_t* c, const double box[3], double sigma, double rcut,
                            const CT* in, CT* tmp, CT* out) {
  const int M[3] = {c->p.size_x, c->p.size_y, c->p.size_z};
  ConvTaps<CT> taps[3];
  conv_taps<CT>(M, box, sigma, rcut, taps);
  CT* rx = (CT*)c->d_rhok;  // the half spectrum holds at least one real grid
  CU(launch_conv_pass<CT>(in, rx, M, 0, taps[0], c->stream));
  CU(launch_conv_pass<CT>(rx, tmp, M, 1, taps[1], c->stream));
  CU(launch_conv_pass<CT>(tmp, out, M, 2, taps[2], c->stream));
  return GSE_OK;
}

}  // namespace

// ===========================================================================
extern "C" {

void gse_params_default(gse_params_t* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->kappa = 0.4;
  p->lambda_sigma = 3.0;
  p->lambda_sigma1 = 3.0;
  p->ccelec = 332.0716;
  p->precision = GSE_PRECISION_FP64;
  p->device = 0;
}

const char* gse_status_string(gse_status_t s) {
  switch (s) {
    case GSE_OK: return "GSE_OK";
    case GSE_ERR_INVALID_ARG: return "GSE_ERR_INVALID_ARG";
    case GSE_ERR_STENCIL_TOO_LARGE: return "GSE_ERR_STENCIL_TOO_LARGE";
    case GSE_ERR_CUDA: return "GSE_ERR_CUDA";
    case GSE_ERR_OOM: return "GSE_ERR_OOM";
    case GSE_ERR_TIMEOUT: return "GSE_ERR_TIMEOUT";
    case GSE_ERR_NOT_READY: return "GSE_ERR_NOT_READY";
    case GSE_ERR_UNSUPPORTED: return "GSE_ERR_UNSUPPORTED";
    case GSE_ERR_NONFINITE: return "GSE_ERR_NONFINITE";
    case GSE_ERR_RANGE: return "GSE_ERR_RANGE";
  }
  return "GSE_ERR_UNKNOWN";
}

const char* gse_last_error(void) { return g_last_error.c_str(); }

int gse_abi_version(void) { return GSE_B200_ABI_VERSION; }

#ifndef GSE_SOURCE_HASH
#define GSE_SOURCE_HASH "unstamped-build"
#endif
// The source hash as a marked string in the library file, where the loader
// reads it without loading the library.
extern "C" __attribute__((used)) const char gse_build_stamp[] =
    "gse-b200-sources:" GSE_SOURCE_HASH;

const char* gse_build_info(void) {
  static char info[128];
  static std::once_flag once;
  std::call_once(once, [] {
    snprintf(info, sizeof(info), "sources %s, nvcc %d.%d.%d, sm_100a", GSE_SOURCE_HASH,
             __CUDACC_VER_MAJOR__, __CUDACC_VER_MINOR__, __CUDACC_VER_BUILD__);
  });
  return info;
}

gse_status_t gse_create(const gse_params_t* params, gse_context_t** out) {
  g_last_error.clear();
  if (!params || !out) return fail(GSE_ERR_INVALID_ARG, "NULL params or out");
  *out = nullptr;
  const gse_params_t& p = *params;
  if (p.size_x < 1 || p.size_y < 1 || p.size_z < 1)
    return fail(GSE_ERR_INVALID_ARG, "grid sizes must be >= 1");
  if ((long long)p.size_x * p.size_y * p.size_z > (1LL << 31) - 1)
    return fail(GSE_ERR_INVALID_ARG, "grid too large for 32-bit FFT plans");
  if (!(p.kappa >= 0.0 && p.kappa <= 0.5))
    return fail(GSE_ERR_INVALID_ARG, "kappa must lie in [0, 0.5] (CpuGSE::setParam)");
  if (!(p.sigma > 0.0) || !(p.box_x > 0.0) || !(p.box_y > 0.0) || !(p.box_z > 0.0) ||
      !(p.lambda_sigma1 > 0.0))
    return fail(GSE_ERR_INVALID_ARG, "sigma, lambda_sigma1 and box lengths must be positive");
  if (p.precision != GSE_PRECISION_FP64 && p.precision != GSE_PRECISION_MIXED)
    return fail(GSE_ERR_INVALID_ARG, "unknown precision %d", p.precision);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(GSE_ERR_UNSUPPORTED, "no CUDA device");
  }
  if (p.device < 0 || p.device >= ndev) return fail(GSE_ERR_INVALID_ARG, "bad device ordinal");
  CU(cudaSetDevice(p.device));
  cudaDeviceProp prop;
  CU(cudaGetDeviceProperties(&prop, p.device));
  if (prop.major != 10)
    return fail(GSE_ERR_UNSUPPORTED, "built for sm_100a; device is sm_%d%d", prop.major,
                prop.minor);

  gse_context_t* c = new gse_context_t();
  c->p = p;
  c->fp64 = (p.precision == GSE_PRECISION_FP64);
  c->ct = c->fp64 ? sizeof(double) : sizeof(float);
  c->sigma1 = p.sigma * std::sqrt(p.kappa);
  c->sigma2 = p.sigma * std::sqrt(1.0 - 2.0 * p.kappa);
  c->rcut1 = p.lambda_sigma1 * std::sqrt(2.0) * c->sigma1;
  c->size = (long long)p.size_x * p.size_y * p.size_z;
  c->ksize = (long long)(p.size_x / 2 + 1) * p.size_y * p.size_z;
  gse_status_t st = check_stencil(c, ctx_box(c).v, c->sigma1, c->rcut1);
  if (st != GSE_OK) {
    delete c;
    return st;
  }
  const int M[3] = {p.size_x, p.size_y, p.size_z};

  auto bail = [&](gse_status_t s) {
    gse_destroy(c);
    return s;
  };
#define CUC(call)                                                                           \
  do {                                                                                      \
    cudaError_t _e = (call);                                                                \
    if (_e != cudaSuccess)                                                                  \
      return bail(fail(_e == cudaErrorMemoryAllocation ? GSE_ERR_OOM : GSE_ERR_CUDA,        \
                       "gse_create: %s: %s", #call, cudaGetErrorString(_e)));               \
  } while (0)
  CUC(cudaMalloc(&c->d_rho, c->size * c->ct));
  CUC(cudaMalloc(&c->d_phi, c->size * c->ct));
  CUC(cudaMalloc(&c->d_rhok, c->ksize * 2 * c->ct));
  if (!c->fp64) CUC(cudaMalloc(&c->d_fixed, c->size * sizeof(long long)));
  {
    const char* env = std::getenv("GSE_B200_OWN_FFT");
    const bool allowed = !(env && env[0] == '0');
    if (!c->fp64 && allowed && own_fft_supported(M)) {
      CUC(make_fft_twiddles(M[0], &c->d_fft_tw));
      c->own_fft = true;
    }
    const char* stall = std::getenv("GSE_B200_TEST_FFT_STALL");
    c->fft_stall_test = stall && stall[0] == '1';
  }
  c->bl = make_bin_layout(M, c->fp64 ? kBinX64 : kBinX32);
  c->nbins2 = bin_count(c->bl);
  CUC(cudaMalloc(&c->d_bcounts, sizeof(int) * c->nbins2));
  CUC(cudaMemset(c->d_bcounts, 0, sizeof(int) * c->nbins2));
  if (!c->fp64) CUC(cudaMalloc(&c->d_blstart, sizeof(int) * c->nbins2));
  CUC(cudaMalloc(&c->d_bstart, sizeof(int) * (c->nbins2 + 1)));
  CUC(cudaMalloc(&c->d_btiles, sizeof(int) * (c->nbins2 / 4096 + 2)));
  CUC(cudaMalloc(&c->d_qmax, sizeof(unsigned)));
  CUC(cudaMalloc(&c->d_partials, sizeof(double) * (kEnergyPartials + 1)));
  CUC(cudaMemset(c->d_partials, 0, sizeof(double) * (kEnergyPartials + 1)));
  CUC(cudaMalloc(&c->d_scalars, sizeof(double) * 16));
  CUC(cudaMalloc(&c->d_bad, sizeof(int)));
  CUC(cudaMemset(c->d_bad, 0, sizeof(int)));
  CUC(cudaMemset(c->d_scalars, 0, sizeof(double) * 16));
  CUC(cudaMallocHost(&c->h_pinned, sizeof(double) * 4));
  {
    int* hb = nullptr;
    CUC(cudaHostAlloc(&hb, sizeof(int), cudaHostAllocMapped));
    *hb = 0;
    c->h_bad = hb;
    CUC(cudaHostGetDevicePointer((void**)&c->d_badmap, hb, 0));
    c->bl.flags = c->d_badmap;
  }
#undef CUC
  if (cufftPlan3d(&c->plan_f, p.size_z, p.size_y, p.size_x, c->fp64 ? CUFFT_D2Z : CUFFT_R2C) !=
          CUFFT_SUCCESS ||
      cufftPlan3d(&c->plan_b, p.size_z, p.size_y, p.size_x, c->fp64 ? CUFFT_Z2D : CUFFT_C2R) !=
          CUFFT_SUCCESS)
    return bail(fail(GSE_ERR_CUDA, "cufftPlan3d failed"));
  c->plans = true;
  if (ensure_atoms(c, 1024) != GSE_OK) return bail(GSE_ERR_OOM);
  *out = c;
  return GSE_OK;
}

gse_status_t gse_destroy(gse_context_t* c) {
  if (!c) return GSE_OK;
  cudaSetDevice(c->p.device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  drop_fwd_graph(c);
  if (c->plans) {
    cufftDestroy(c->plan_f);
    cufftDestroy(c->plan_b);
  }
  if (c->green_cb) cufftDestroy(c->plan_bg);
  cudaFree(c->d_rho);
  cudaFree(c->d_phi);
  cudaFree(c->d_rhok);
  cudaFree(c->d_fft_tw);
  cudaFree(c->d_scratch);
  cudaFree(c->d_fixed);
  cudaFree(c->d_xyzq);
  cudaFree(c->d_sorted);
  cudaFree(c->d_perm);
  cudaFree(c->d_force);
  cudaFree(c->d_bkey);
  cudaFree(c->d_btmp);
  cudaFree(c->d_bcounts);
  cudaFree(c->d_blstart);
  cudaFree(c->d_bstart);
  cudaFree(c->d_btiles);
  cudaFree(c->d_qmax);
  cudaFree(c->d_gtab);
  cudaFree(c->d_adj);
  cudaFree(c->d_partials);
  cudaFree(c->d_scalars);
  cudaFree(c->d_bad);
  if (c->h_bad) cudaFreeHost((void*)c->h_bad);
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  for (int i = 0; i < GSE_NUM_STAGES; i++)
    for (int j = 0; j < 2; j++)
      if (c->ev[i][j]) cudaEventDestroy(c->ev[i][j]);
  delete c;
  return GSE_OK;
}

gse_status_t gse_set_stream(gse_context_t* c, void* stream) {
  TRY(check_ctx(c));
  drop_fwd_graph(c);
  c->stream = (cudaStream_t)stream;
  CUFFT(cufftSetStream(c->plan_f, c->stream));
  CUFFT(cufftSetStream(c->plan_b, c->stream));
  if (c->green_cb) CUFFT(cufftSetStream(c->plan_bg, c->stream));
  return GSE_OK;
}

gse_status_t gse_set_box(gse_context_t* c, double bx, double by, double bz) {
  TRY(check_ctx(c));
  if (!(bx > 0.0 && by > 0.0 && bz > 0.0)) return fail(GSE_ERR_INVALID_ARG, "box must be > 0");
  const gse_params_t old = c->p;
  c->p.box_x = bx;
  c->p.box_y = by;
  c->p.box_z = bz;
  gse_status_t s = check_stencil(c, ctx_box(c).v, c->sigma1, c->rcut1);
  if (s != GSE_OK) {
    c->p = old;
    return s;
  }
  c->phi_valid = c->energy_valid = false;
  c->gtab_valid = false;
  return GSE_OK;
}

gse_status_t gse_synchronize(gse_context_t* c) {
  TRY(check_ctx(c));
  CU(cudaStreamSynchronize(c->stream));
  return check_finite(c);
}

gse_status_t gse_spread_charge(gse_context_t* c, int n, const void* xyzq) {
  TRY(check_ctx(c));
  const void* dx;
  TRY(stage_atoms(c, n, xyzq, &dx));
  if (c->fp64)
    TRY(do_spread<double>(c, n, dx, ctx_box(c).v, c->sigma1, c->rcut1, false));
  else
    TRY(do_spread<float>(c, n, dx, ctx_box(c).v, c->sigma1, c->rcut1, false));
  return finish(c, false);
}

gse_status_t gse_solve_poisson(gse_context_t* c) {
  TRY(check_ctx(c));
  if (!c->rho_valid) return fail(GSE_ERR_NOT_READY, "solvePoisson before spreadCharge1");
  TRY(do_solve_ctx(c));
  c->phi_valid = true;
  c->energy_valid = true;
  return finish(c, false);
}

gse_status_t gse_calculate_energy(gse_context_t* c, double* energy) {
  TRY(check_ctx(c));
  if (!energy) return fail(GSE_ERR_INVALID_ARG, "NULL energy");
  TRY(check_ptr(energy, c->p.device, 1, "energy"));
  if (!c->rho_valid || !c->phi_valid)
    return fail(GSE_ERR_NOT_READY, "calculateEnergy needs rhoS and phiM");
  if (!c->energy_valid) {
    if (c->fp64)
      CU(launch_dot_energy<double>((const double*)c->d_rho, (const double*)c->d_phi, c->size,
                                   c->d_partials, kEnergyPartials, energy_factor(c),
                                   c->d_scalars, c->stream));
    else
      CU(launch_dot_energy<float>((const float*)c->d_rho, (const float*)c->d_phi, c->size,
                                  c->d_partials, kEnergyPartials, energy_factor(c), c->d_scalars,
                                  c->stream));
    c->energy_valid = true;
  }
  bool host = false;
  TRY(energy_out(c, energy, &host));
  return finish(c, host);
}

gse_status_t gse_interpolate_force(gse_context_t* c, int n, const void* xyzq, double* fx,
                                   double* fy, double* fz) {
  TRY(check_ctx(c));
  if (n > 0 && (!fx || !fy || !fz)) return fail(GSE_ERR_INVALID_ARG, "NULL force array");
  TRY(check_xyz(c->p.device, fx, fy, fz, "force array"));
  if (!c->phi_valid) return fail(GSE_ERR_NOT_READY, "interpolateForce before solvePoisson");
  const void* dx;
  TRY(stage_atoms(c, n, xyzq, &dx));
  bool host = false;
  if (c->fp64)
    TRY(gather_to<double>(c, n, dx, ctx_box(c).v, c->sigma1, c->rcut1, (const double*)c->d_phi, c->p.ccelec,
                          fx, fy, fz, &host));
  else
    TRY(gather_to<float>(c, n, dx, ctx_box(c).v, c->sigma1, c->rcut1, (const float*)c->d_phi, c->p.ccelec, fx,
                         fy, fz, &host));
  return finish(c, host);
}

gse_status_t gse_interpolate_field(gse_context_t* c, int n, const void* xyzq, double* ex,
                                   double* ey, double* ez) {
  TRY(check_ctx(c));
  if (n > 0 && (!ex || !ey || !ez)) return fail(GSE_ERR_INVALID_ARG, "NULL field array");
  TRY(check_xyz(c->p.device, ex, ey, ez, "field array"));
  if (!c->phi_valid) return fail(GSE_ERR_NOT_READY, "field before solvePoisson");
  const void* dx;
  TRY(stage_atoms(c, n, xyzq, &dx));
  // unit charges in the context's own atom buffer (a host input is already there)
  c->launches += n > 0 ? 1 : 0;
  if (c->fp64)
    CU(launch_unit_charges<double>((const double4*)dx, (double4*)c->d_xyzq, n, c->stream));
  else
    CU(launch_unit_charges<float>((const float4*)dx, (float4*)c->d_xyzq, n, c->stream));
  bool host = false;
  if (c->fp64)
    TRY(gather_to<double>(c, n, c->d_xyzq, ctx_box(c).v, c->sigma1, c->rcut1,
                          (const double*)c->d_phi, c->p.ccelec, ex, ey, ez, &host));
  else
    TRY(gather_to<float>(c, n, c->d_xyzq, ctx_box(c).v, c->sigma1, c->rcut1,
                         (const float*)c->d_phi, c->p.ccelec, ex, ey, ez, &host));
  return finish(c, host);
}

// The four forward calls in one pass (sorting once for spread and gather).
gse_status_t forward_body(gse_context_t* c, int n, const void* xyzq, double* energy, double* fx,
                          double* fy, double* fz, bool* host) {
  const void* dx = nullptr;
  TRY(stage_atoms(c, n, xyzq, &dx));
  const Box3 box = ctx_box(c);
  // one stable sort serves the spread and the gather; the mixed form's
  // counting kernel clears the int64 grid on the way, so that the spread
  // follows the binning directly (a memset in the spread stage when stages
  // are timed)
  bool zeroed = false;
  if (c->fp64) {
    TRY(bin_atoms<double>(c, n, dx, stencil_of<double>(c, box.v, c->sigma1, c->rcut1, false, false)));
  } else {
    const Stencil<float> s = stencil_of<float>(c, box.v, c->sigma1, c->rcut1, false, false);
    zeroed = !c->timing && tiled_ok<float>(c, s);
    TRY(bin_atoms<float>(c, n, dx, s, zeroed));
  }
  if (c->fp64)
    TRY(do_spread<double>(c, n, dx, box.v, c->sigma1, c->rcut1, false, true));
  else
    TRY(do_spread<float>(c, n, dx, box.v, c->sigma1, c->rcut1, false, true, true, zeroed));
  TRY(do_solve_ctx(c));
  c->phi_valid = true;
  c->energy_valid = true;
  if (fx || fy || fz) {
    if (c->fp64)
      TRY(gather_to<double>(c, n, dx, box.v, c->sigma1, c->rcut1, (const double*)c->d_phi,
                            c->p.ccelec, fx, fy, fz, host, true));
    else
      TRY(gather_to<float>(c, n, dx, box.v, c->sigma1, c->rcut1, (const float*)c->d_phi,
                           c->p.ccelec, fx, fy, fz, host, true, true));
  }
  return energy_out(c, energy, host);
}

gse_status_t gse_forward(gse_context_t* c, int n, const void* xyzq, double* energy, double* fx,
                         double* fy, double* fz) {
  TRY(check_ctx(c));
  // A repeat of the captured call (same count, positions, forces, box and
  // stream) replays its graph: its pointers were checked and classified when
  // it was captured.  Only a host energy may change address between calls.
  const gse_context_t::FwdKey& k = c->fwd_key;
  if (c->fwd_exec && !c->timing && n == k.n && xyzq == k.x && fx == k.fx && fy == k.fy &&
      fz == k.fz && c->stream == k.stream && c->p.box_x == k.box[0] && c->p.box_y == k.box[1] &&
      c->p.box_z == k.box[2]) {
    bool he = c->fwd_e_host;
    if (energy != c->fwd_e_raw) {
      TRY(check_ptr(energy, c->p.device, 1, "energy"));
      he = energy && !is_device_ptr(energy);
    }
    if ((he ? reinterpret_cast<double*>(uintptr_t(1)) : energy) == k.e) {
      CU(cudaGraphLaunch(c->fwd_exec, c->stream));
      c->launches += c->fwd_launches;
      c->rho_valid = c->phi_valid = c->energy_valid = true;
      c->fwd_e_raw = energy;
      c->fwd_e_host = he;
      TRY(finish(c, c->fwd_host_io));
      if (he) *energy = c->h_pinned[0];
      return GSE_OK;
    }
  }
  TRY(check_ptr(xyzq, c->p.device, 4 * c->ct, "xyzq"));
  TRY(check_ptr(energy, c->p.device, 1, "energy"));
  TRY(check_xyz(c->p.device, fx, fy, fz, "force array"));
  // Graph replay applies to calls whose positions and forces are device or
  // page-locked host memory (the copies to and from the host then sit in the
  // graph), on a stream that can be captured, without stage timing; the key
  // (pointers, count, box, stream) must repeat exactly.  A host energy is read
  // through the context's page-locked scalar after the call has finished.
  auto io_ok = [](const void* p) { return is_device_ptr(p) || is_pinned_host(p); };
  const bool host_e = energy && !is_device_ptr(energy);
  const bool forces_ok = (!fx && !fy && !fz) || (fx && fy && fz && io_ok(fx) && io_ok(fy) &&
                                                 io_ok(fz));
  const bool host_io = host_e || (fx && !is_device_ptr(fx)) || (fy && !is_device_ptr(fy)) ||
                       (fz && !is_device_ptr(fz));
  const bool graphable = c->fwd_graphs && !c->timing && c->stream != nullptr && n > 0 &&
                         io_ok(xyzq) && forces_ok && c->gtab_valid;
  gse_context_t::FwdKey key;
  key.n = n;
  key.x = xyzq;
  // a host energy is not part of the graph (it is read from the scalar after
  // the call), so its address need not repeat
  key.e = host_e ? reinterpret_cast<double*>(uintptr_t(1)) : energy;
  key.fx = fx;
  key.fy = fy;
  key.fz = fz;
  key.box[0] = c->p.box_x;
  key.box[1] = c->p.box_y;
  key.box[2] = c->p.box_z;
  key.stream = c->stream;
  bool host = false;
  if (!graphable) {
    drop_fwd_graph(c);
    TRY(forward_body(c, n, xyzq, energy, fx, fy, fz, &host));
    return finish(c, host);
  }
  // the evaluation with the energy copied to the page-locked scalar, no wait
  auto body = [&](bool* h) -> gse_status_t {
    TRY(forward_body(c, n, xyzq, host_e ? nullptr : energy, fx, fy, fz, h));
    if (host_e) {
      CU(cudaMemcpyAsync(c->h_pinned, c->d_scalars, sizeof(double), cudaMemcpyDeviceToHost,
                         c->stream));
      *h = true;
    }
    return GSE_OK;
  };
  auto done = [&](bool h) -> gse_status_t {
    TRY(finish(c, h));
    if (host_e) *energy = c->h_pinned[0];
    return GSE_OK;
  };
  if (c->fwd_exec && key == c->fwd_key) {
    CU(cudaGraphLaunch(c->fwd_exec, c->stream));
    c->launches += c->fwd_launches;
    c->rho_valid = c->phi_valid = c->energy_valid = true;
    return done(host_io);
  }
  if (!(key == c->fwd_key)) {
    // first call with this key: run it directly and remember the key
    drop_fwd_graph(c);
    TRY(body(&host));
    c->fwd_key = key;
    return done(host);
  }
  // second identical call: capture, instantiate, launch
  const long long l0 = c->launches;
  CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  const gse_status_t st = body(&host);
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
  gse_status_t result = st;
  if (st == GSE_OK && ec == cudaSuccess) {
    const cudaError_t ei = cudaGraphInstantiate(&c->fwd_exec, g, 0);
    if (ei == cudaSuccess) {
      c->fwd_launches = c->launches - l0;
      c->fwd_host_io = host_io;
      c->fwd_e_host = host_e;
      c->fwd_e_raw = energy;
      const cudaError_t el = cudaGraphLaunch(c->fwd_exec, c->stream);
      if (el != cudaSuccess) result = fail(GSE_ERR_CUDA, "cudaGraphLaunch: %s", cudaGetErrorString(el));
    } else {
      c->fwd_exec = nullptr;
    }
  }
  if (g) cudaGraphDestroy(g);
  if (!c->fwd_exec || result != GSE_OK) {
    // capture failed: this pass ran nothing, so run it directly and stop trying
    cudaGetLastError();
    c->fwd_graphs = false;
    drop_fwd_graph(c);
    c->launches = l0;
    host = false;
    TRY(body(&host));
  }
  return done(host);
}

gse_status_t gse_get_grid(gse_context_t* c, int which, void* out) {
  TRY(check_ctx(c));
  if (!out) return fail(GSE_ERR_INVALID_ARG, "NULL out");
  TRY(check_ptr(out, c->p.device, 1, "out"));
  const void* src;
  if (which == GSE_GRID_RHO) {
    if (!c->rho_valid) return fail(GSE_ERR_NOT_READY, "rhoS not computed");
    src = c->d_rho;
  } else if (which == GSE_GRID_PHI) {
    if (!c->phi_valid) return fail(GSE_ERR_NOT_READY, "phiM not computed");
    src = c->d_phi;
  } else {
    return fail(GSE_ERR_INVALID_ARG, "unknown grid id %d", which);
  }
  bool host = false;
  TRY(copy_out(c, out, src, c->size * c->ct, &host));
  return finish(c, host);
}

gse_status_t gse_set_grid(gse_context_t* c, int which, const void* in) {
  TRY(check_ctx(c));
  if (!in) return fail(GSE_ERR_INVALID_ARG, "NULL in");
  TRY(check_ptr(in, c->p.device, 1, "in"));
  void* dst;
  if (which == GSE_GRID_RHO)
    dst = c->d_rho;
  else if (which == GSE_GRID_PHI)
    dst = c->d_phi;
  else
    return fail(GSE_ERR_INVALID_ARG, "unknown grid id %d", which);
  CU(cudaMemcpyAsync(dst, in, c->size * c->ct,
                     is_device_ptr(in) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     c->stream));
  if (which == GSE_GRID_RHO) {
    c->rho_valid = true;
    c->phi_valid = false;
  } else {
    c->phi_valid = true;
  }
  c->energy_valid = false;
  return finish(c, true);
}

gse_status_t gse_gauss_spread(gse_context_t* c, double sigma, double rcut, int n,
                              const void* xyzq, double bx, double by, double bz, int normalize,
                              void* rho_out) {
  TRY(check_ctx(c));
  TRY(check_ptr(xyzq, c->p.device, 4 * c->ct, "xyzq"));
  TRY(check_ptr(rho_out, c->p.device, 1, "rho_out"));
  const double box[3] = {bx, by, bz};
  TRY(check_stencil(c, box, sigma, rcut));
  const void* dx;
  TRY(stage_atoms(c, n, xyzq, &dx));
  if (c->fp64)
    TRY(do_spread<double>(c, n, dx, box, sigma, rcut, normalize != 0));
  else
    TRY(do_spread<float>(c, n, dx, box, sigma, rcut, normalize != 0));
  bool host = false;
  if (rho_out && rho_out != c->d_rho) TRY(copy_out(c, rho_out, c->d_rho, c->size * c->ct, &host));
  return finish(c, host);
}

gse_status_t gse_gauss_interpolate(gse_context_t* c, double sigma, double rcut, int n,
                                   const void* xyzq, double bx, double by, double bz,
                                   const void* phi, double* fx, double* fy, double* fz) {
  TRY(check_ctx(c));
  if (!phi) return fail(GSE_ERR_INVALID_ARG, "NULL phi");
  if (n > 0 && (!fx || !fy || !fz)) return fail(GSE_ERR_INVALID_ARG, "NULL force array");
  TRY(check_ptr(xyzq, c->p.device, 4 * c->ct, "xyzq"));
  TRY(check_ptr(phi, c->p.device, c->ct, "phi"));
  TRY(check_xyz(c->p.device, fx, fy, fz, "force array"));
  const double box[3] = {bx, by, bz};
  TRY(check_stencil(c, box, sigma, rcut));
  const void* dphi = phi;
  if (!is_device_ptr(phi)) {
    CU(cudaMemcpyAsync(c->d_phi, phi, c->size * c->ct, cudaMemcpyHostToDevice, c->stream));
    c->phi_valid = true;
    c->energy_valid = false;
    dphi = c->d_phi;
  }
  const void* dx;
  TRY(stage_atoms(c, n, xyzq, &dx));
  bool host = false;
  if (c->fp64)
    TRY(gather_to<double>(c, n, dx, box, sigma, rcut, (const double*)dphi, 1.0, fx, fy, fz, &host));
  else
    TRY(gather_to<float>(c, n, dx, box, sigma, rcut, (const float*)dphi, 1.0, fx, fy, fz, &host));
  return finish(c, host);
}

gse_status_t gse_green_mul(gse_context_t* c, double sigma, double bx, double by, double bz,
                           void* rho_k) {
  TRY(check_ctx(c));
  if (!rho_k) return fail(GSE_ERR_INVALID_ARG, "NULL rho_k");
  TRY(check_ptr(rho_k, c->p.device, 16, "rho_k"));
  if (!(sigma >= 0.0) || !(bx > 0 && by > 0 && bz > 0))
    return fail(GSE_ERR_INVALID_ARG, "bad sigma or box");
  const bool dev = is_device_ptr(rho_k);
  void* k = dev ? rho_k : c->d_rhok;
  const size_t bytes = c->ksize * 2 * c->ct;
  if (!dev) CU(cudaMemcpyAsync(k, rho_k, bytes, cudaMemcpyHostToDevice, c->stream));
  const GreenGeom g = green_geom(c, sigma, bx, by, bz, false);
  if (c->fp64)
    CU(launch_green_energy<double>((double2*)k, g, c->d_partials, kEnergyPartials, 1.0,
                                   c->d_scalars + 1, c->stream));
  else
    CU(launch_green_energy<float>((float2*)k, g, c->d_partials, kEnergyPartials, 1.0,
                                  c->d_scalars + 1, c->stream));
  bool host = false;
  if (!dev) TRY(copy_out(c, rho_k, k, bytes, &host));
  return finish(c, host);
}

gse_status_t gse_fft_solve(gse_context_t* c, double sigma, double bx, double by, double bz,
                           const void* rho, void* phi) {
  TRY(check_ctx(c));
  if (!rho || !phi) return fail(GSE_ERR_INVALID_ARG, "NULL grid");
  TRY(check_ptr(rho, c->p.device, 16, "rho"));
  TRY(check_ptr(phi, c->p.device, 16, "phi"));
  if (!(sigma >= 0.0) || !(bx > 0 && by > 0 && bz > 0))
    return fail(GSE_ERR_INVALID_ARG, "bad sigma or box");
  const size_t bytes = c->size * c->ct;
  const void* drho = rho;
  if (!is_device_ptr(rho)) {
    CU(cudaMemcpyAsync(c->d_rho, rho, bytes, cudaMemcpyHostToDevice, c->stream));
    drho = c->d_rho;
    c->rho_valid = true;
  }
  const bool pdev = is_device_ptr(phi);
  void* dphi = pdev ? phi : c->d_phi;
  TRY(do_solve(c, drho, dphi, sigma, bx, by, bz, false));
  if (dphi == c->d_phi) c->phi_valid = true;
  c->energy_valid = false;
  bool host = false;
  if (!pdev) TRY(copy_out(c, phi, c->d_phi, bytes, &host));
  return finish(c, host);
}

// ---- grid operations beside the force path -------------------------------

gse_status_t gse_gauss_spread_on_grid(gse_context_t* c, double sigma, double rcut, double bx,
                                      double by, double bz, const void* rho, void* rho_s) {
  TRY(check_ctx(c));
  if (!rho || !rho_s) return fail(GSE_ERR_INVALID_ARG, "NULL grid");
  TRY(check_ptr(rho, c->p.device, c->ct, "rho"));
  TRY(check_ptr(rho_s, c->p.device, c->ct, "rho_s"));
  const double box[3] = {bx, by, bz};
  TRY(check_stencil(c, box, sigma, rcut));
  const size_t bytes = c->size * c->ct;
  TRY(ensure_scratch(c, bytes));
  const void* in = rho;
  if (!is_device_ptr(rho)) {
    CU(cudaMemcpyAsync(c->d_scratch, rho, bytes, cudaMemcpyHostToDevice, c->stream));
    in = c->d_scratch;
  }
  // the x pass reads the input before the z pass writes the output, so the
  // two may be the same device grid
  const bool odev = is_device_ptr(rho_s);
  void* out = odev ? rho_s : c->d_rho;
  if (c->fp64)
    TRY(spread_on_grid<double>(c, box, sigma, rcut, (const double*)in, (double*)c->d_scratch,
                               (double*)out));
  else
    TRY(spread_on_grid<float>(c, box, sigma, rcut, (const float*)in, (float*)c->d_scratch,
                              (float*)out));
  if (out == c->d_rho) {
    c->rho_valid = true;
    c->phi_valid = false;
    c->energy_valid = false;
  }
  bool host = false;
  if (!odev) TRY(copy_out(c, rho_s, c->d_rho, bytes, &host));
  return finish(c, host);
}

gse_status_t gse_gauss_efield_on_grid(gse_context_t* c, double bx, double by, double bz,
                                      const void* phi, void* ex, void* ey, void* ez) {
  TRY(check_ctx(c));
  if (!phi || !ex || !ey || !ez) return fail(GSE_ERR_INVALID_ARG, "NULL grid");
  TRY(check_ptr(phi, c->p.device, c->ct, "phi"));
  TRY(check_ptr(ex, c->p.device, c->ct, "ex"));
  TRY(check_ptr(ey, c->p.device, c->ct, "ey"));
  TRY(check_ptr(ez, c->p.device, c->ct, "ez"));
  if (!(bx > 0 && by > 0 && bz > 0) || !std::isfinite(bx) || !std::isfinite(by) ||
      !std::isfinite(bz))
    return fail(GSE_ERR_INVALID_ARG, "box lengths must be positive and finite");
  const int M[3] = {c->p.size_x, c->p.size_y, c->p.size_z};
  const size_t bytes = c->size * c->ct;
  void* outs[3] = {ex, ey, ez};
  bool odev[3];
  int nhost = 0;
  for (int d = 0; d < 3; d++) {
    odev[d] = is_device_ptr(outs[d]);
    if (!odev[d]) nhost++;
  }
  const bool idev = is_device_ptr(phi);
  TRY(ensure_scratch(c, bytes * ((idev ? 0 : 1) + nhost)));
  char* sp = (char*)c->d_scratch;
  const void* in = phi;
  if (!idev) {
    CU(cudaMemcpyAsync(sp, phi, bytes, cudaMemcpyHostToDevice, c->stream));
    in = sp;
    sp += bytes;
  }
  void* dst[3];
  for (int d = 0; d < 3; d++) {
    if (odev[d]) {
      dst[d] = outs[d];
    } else {
      dst[d] = sp;
      sp += bytes;
    }
  }
  const double hd[3] = {bx / (double)M[0], by / (double)M[1], bz / (double)M[2]};
  if (c->fp64) {
    const double ih[3] = {1.0 / hd[0], 1.0 / hd[1], 1.0 / hd[2]};
    CU(launch_efield<double>((const double*)in, (double*)dst[0], (double*)dst[1], (double*)dst[2],
                             M, ih, c->stream));
  } else {
    const float ih[3] = {(float)(1.0 / hd[0]), (float)(1.0 / hd[1]), (float)(1.0 / hd[2])};
    CU(launch_efield<float>((const float*)in, (float*)dst[0], (float*)dst[1], (float*)dst[2], M,
                            ih, c->stream));
  }
  bool host = false;
  for (int d = 0; d < 3; d++)
    if (!odev[d]) TRY(copy_out(c, outs[d], dst[d], bytes, &host));
  return finish(c, host);
}

gse_status_t gse_gauss_dipole_sum(gse_context_t* c, double bx, double by, double bz,
                                  const void* rho, double* dip) {
  TRY(check_ctx(c));
  if (!rho || !dip) return fail(GSE_ERR_INVALID_ARG, "NULL argument");
  TRY(check_ptr(rho, c->p.device, c->ct, "rho"));
  TRY(check_ptr(dip, c->p.device, 1, "dip"));
  if (!(bx > 0 && by > 0 && bz > 0) || !std::isfinite(bx) || !std::isfinite(by) ||
      !std::isfinite(bz))
    return fail(GSE_ERR_INVALID_ARG, "box lengths must be positive and finite");
  const int M[3] = {c->p.size_x, c->p.size_y, c->p.size_z};
  const size_t bytes = c->size * c->ct;
  const void* in = rho;
  if (!is_device_ptr(rho)) {
    TRY(ensure_scratch(c, bytes));
    CU(cudaMemcpyAsync(c->d_scratch, rho, bytes, cudaMemcpyHostToDevice, c->stream));
    in = c->d_scratch;
  }
  static_assert(3 * kDipoleBlocks <= kEnergyPartials, "dipole partials fit the energy partials");
  unsigned* done = reinterpret_cast<unsigned*>(c->d_partials + kEnergyPartials);
  double* out = c->d_scalars + 4;
  if (c->fp64) {
    const double h[3] = {bx / (double)M[0], by / (double)M[1], bz / (double)M[2]};
    CU(launch_dipole<double>((const double*)in, M, h, c->d_partials, done, out, c->stream));
  } else {
    const float h[3] = {(float)(bx / (double)M[0]), (float)(by / (double)M[1]),
                        (float)(bz / (double)M[2])};
    CU(launch_dipole<float>((const float*)in, M, h, c->d_partials, done, out, c->stream));
  }
  bool host = false;
  TRY(copy_out(c, dip, out, 3 * sizeof(double), &host));
  return finish(c, host);
}

gse_status_t gse_virial(gse_context_t* c, double* virial) {
  TRY(check_ctx(c));
  if (!virial) return fail(GSE_ERR_INVALID_ARG, "NULL virial");
  TRY(check_ptr(virial, c->p.device, 1, "virial"));
  if (!c->rho_valid) return fail(GSE_ERR_NOT_READY, "virial needs rhoS (spread or forward first)");
  if (c->fixed_pending) {
    CU(launch_grid64_to_real(c->d_fixed, c->size, (float*)c->d_rho, c->stream));
    c->fixed_pending = false;
  }
  const GreenGeom g = green_geom(c, c->sigma2, c->p.box_x, c->p.box_y, c->p.box_z, false);
  if (!c->d_gtab) CU(cudaMalloc(&c->d_gtab, c->ksize * c->ct));
  if (!c->gtab_valid) {
    if (c->fp64)
      CU(launch_green_table<double>(g, (double*)c->d_gtab, c->stream));
    else
      CU(launch_green_table<float>(g, (float*)c->d_gtab, c->stream));
    c->gtab_valid = true;
  }
  TRY(fft_forward(c, c->d_rho, c->d_rhok));
  const int nb = std::min(sm_count() * 2, kEnergyPartials / 6);
  unsigned* done = reinterpret_cast<unsigned*>(c->d_partials + kEnergyPartials);
  const double hs2 = 0.5 * c->p.sigma * c->p.sigma;
  double* out = c->d_scalars + 8;
  c->launches += 1;
  if (c->fp64)
    CU(launch_virial<double>((const double2*)c->d_rhok, (const double*)c->d_gtab, g, hs2,
                             energy_factor(c), c->d_partials, done, nb, out, c->stream));
  else
    CU(launch_virial<float>((const float2*)c->d_rhok, (const float*)c->d_gtab, g, hs2,
                            energy_factor(c), c->d_partials, done, nb, out, c->stream));
  bool host = false;
  TRY(copy_out(c, virial, out, 6 * sizeof(double), &host));
  return finish(c, host);
}

gse_status_t gse_set_timing(gse_context_t* c, int enable) {
  TRY(check_ctx(c));
  if (enable && !c->ev[0][0]) {
    for (int i = 0; i < GSE_NUM_STAGES; i++)
      for (int j = 0; j < 2; j++) CU(cudaEventCreate(&c->ev[i][j]));
  }
  if (!enable && c->timing) {
    CU(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < GSE_NUM_STAGES; i++) harvest(c, i);
  }
  c->timing = enable != 0;
  return GSE_OK;
}

gse_status_t gse_get_paths(gse_context_t* c, int* flags) {
  TRY(check_ctx(c));
  if (!flags) return fail(GSE_ERR_INVALID_ARG, "NULL flags");
  const Box3 box = ctx_box(c);
  int f = 0;
  if (c->fp64 ? tiled_ok<double>(c, stencil_of<double>(c, box.v, c->sigma1, c->rcut1, false, false))
              : tiled_ok<float>(c, stencil_of<float>(c, box.v, c->sigma1, c->rcut1, false, false)))
    f |= GSE_PATH_TILED;
  if (c->green_cb) f |= GSE_PATH_GREEN_IN_FFT;
  if (c->own_fft) f |= GSE_PATH_OWN_FFT;
  if (c->fwd_exec) f |= GSE_PATH_GRAPH;
  *flags = f;
  return GSE_OK;
}

gse_status_t gse_get_launch_count(gse_context_t* c, long long* launches) {
  TRY(check_ctx(c));
  if (!launches) return fail(GSE_ERR_INVALID_ARG, "NULL launches");
  *launches = c->launches;
  return GSE_OK;
}

gse_status_t gse_get_timing(gse_context_t* c, double* ms_total, long long* counts, int reset) {
  TRY(check_ctx(c));
  CU(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < GSE_NUM_STAGES; i++) {
    harvest(c, i);
    if (ms_total) ms_total[i] = c->stage_ms[i];
    if (counts) counts[i] = c->stage_count[i];
    if (reset) {
      c->stage_ms[i] = 0.0;
      c->stage_count[i] = 0;
    }
  }
  return GSE_OK;
}

gse_status_t gse_adjoint(gse_context_t* c, int n, const void* xyzq, double dLdE,
                         const double* gfx, const double* gfy, const double* gfz, double* dq,
                         double* dx, double* dy, double* dz) {
  TRY(check_ctx(c));
  if (n > 0 && (!dq || !dx || !dy || !dz)) return fail(GSE_ERR_INVALID_ARG, "NULL output");
  const bool have_g = gfx || gfy || gfz;
  if (have_g && !(gfx && gfy && gfz))
    return fail(GSE_ERR_INVALID_ARG, "force gradients: give all three components or none");
  TRY(check_ptr(xyzq, c->p.device, 4 * c->ct, "xyzq"));
  TRY(check_xyz(c->p.device, gfx, gfy, gfz, "force gradient"));
  TRY(check_ptr(dq, c->p.device, sizeof(double), "dq"));
  TRY(check_xyz(c->p.device, dx, dy, dz, "position gradient"));
  const void* dxq;
  TRY(stage_atoms(c, n, xyzq, &dxq));
  if (n == 0) return finish(c, false);
  if (c->adj_cap < c->atom_cap) {
    cudaFree(c->d_adj);
    c->d_adj = nullptr;
    c->adj_cap = 0;
    CU(cudaMalloc(&c->d_adj, 7 * c->atom_cap * sizeof(double)));
    c->adj_cap = c->atom_cap;
  }
  const size_t cap = c->adj_cap;
  double* g = c->d_adj;           // upstream dL/dF (3 x cap)
  double* o = c->d_adj + 3 * cap; // dq, dx, dy, dz (4 x cap)
  const double* gd[3] = {nullptr, nullptr, nullptr};
  if (have_g) {
    const double* gin[3] = {gfx, gfy, gfz};
    for (int d = 0; d < 3; d++) {
      if (is_device_ptr(gin[d])) {
        gd[d] = gin[d];
      } else {
        CU(cudaMemcpyAsync(g + d * cap, gin[d], n * sizeof(double), cudaMemcpyHostToDevice,
                           c->stream));
        gd[d] = g + d * cap;
      }
    }
  } else {
    CU(cudaMemsetAsync(g, 0, 3 * cap * sizeof(double), c->stream));
    for (int d = 0; d < 3; d++) gd[d] = g + d * cap;
  }
  const Box3 box = ctx_box(c);
  const double h3 = (c->p.box_x / c->p.size_x) * (c->p.box_y / c->p.size_y) *
                    (c->p.box_z / c->p.size_z);
  const double gE_ch3 = dLdE * c->p.ccelec * h3;
  // forward grids, recomputed from the inputs (rho -> phi)
  if (c->fp64)
    TRY(bin_atoms<double>(c, n, dxq, stencil_of<double>(c, box.v, c->sigma1, c->rcut1, false, false)));
  else
    TRY(bin_atoms<float>(c, n, dxq, stencil_of<float>(c, box.v, c->sigma1, c->rcut1, false, false)));
  if (c->fp64)
    TRY(do_spread<double>(c, n, dxq, box.v, c->sigma1, c->rcut1, false, true));
  else
    TRY(do_spread<float>(c, n, dxq, box.v, c->sigma1, c->rcut1, false, true));
  TRY(do_solve_ctx(c));
  c->phi_valid = true;
  c->energy_valid = true;
  // adjoint source lambda into the rho buffer, then psi = K lambda in place
  const bool tiled_mixed =
      !c->fp64 && tiled_ok<float>(c, stencil_of<float>(c, box.v, c->sigma1, c->rcut1, true, false));
  if (tiled_mixed) {
    const Stencil<float> sg = stencil_of<float>(c, box.v, c->sigma1, c->rcut1, true, false);
    c->launches += 2;
    CU(launch_adj_scatter((const float4*)c->d_sorted, c->d_perm, c->d_bstart, c->bl, sg,
                          c->p.ccelec, gd[0], gd[1], gd[2], c->d_fixed, (float*)c->d_rho,
                          c->stream));
  } else {
  CU(cudaMemsetAsync(c->d_rho, 0, c->size * c->ct, c->stream));
  c->launches += 3;
  if (c->fp64) {
    const Stencil<double> sg = stencil_of<double>(c, box.v, c->sigma1, c->rcut1, true, false);
    CU(launch_adj_source<double>((const double4*)c->d_sorted, c->d_perm, n, sg, c->p.ccelec,
                                 gd[0], gd[1], gd[2], (double*)c->d_rho, c->stream));
  } else {
    const Stencil<float> sg = stencil_of<float>(c, box.v, c->sigma1, c->rcut1, true, false);
    CU(launch_adj_source<float>((const float4*)c->d_sorted, c->d_perm, n, sg, c->p.ccelec, gd[0],
                                gd[1], gd[2], (float*)c->d_rho, c->stream));
  }
  }
  TRY(do_solve(c, c->d_rho, c->d_rho, c->sigma2, c->p.box_x, c->p.box_y, c->p.box_z, false));
  c->rho_valid = false;
  const bool dev_out = is_device_ptr(dq) && is_device_ptr(dx) && is_device_ptr(dy) &&
                       is_device_ptr(dz);
  double* od[4];
  if (dev_out) {
    od[0] = dq; od[1] = dx; od[2] = dy; od[3] = dz;
  } else {
    for (int k = 0; k < 4; k++) od[k] = o + k * cap;
  }
  if (tiled_mixed) {
    const Stencil<float> sp = stencil_of<float>(c, box.v, c->sigma1, c->rcut1, false, false);
    const Stencil<float> sg = stencil_of<float>(c, box.v, c->sigma1, c->rcut1, true, false);
    c->launches += 1;
    CU(launch_adj_gather_tiled((const float4*)c->d_sorted, c->d_perm, c->d_bstart, c->bl, sp, sg,
                               c->p.ccelec, gE_ch3, (const float*)c->d_rho,
                               (const float*)c->d_phi, gd[0], gd[1], gd[2], od[0], od[1], od[2],
                               od[3], c->stream));
  } else if (c->fp64) {
    const Stencil<double> sp = stencil_of<double>(c, box.v, c->sigma1, c->rcut1, false, false);
    const Stencil<double> sg = stencil_of<double>(c, box.v, c->sigma1, c->rcut1, true, false);
    CU(launch_adj_gather<double>((const double4*)c->d_sorted, c->d_perm, n, sp, sg, c->p.ccelec,
                                 gE_ch3, (const double*)c->d_rho, (const double*)c->d_phi, gd[0],
                                 gd[1], gd[2], od[0], od[1], od[2], od[3], c->stream));
  } else {
    const Stencil<float> sp = stencil_of<float>(c, box.v, c->sigma1, c->rcut1, false, false);
    const Stencil<float> sg = stencil_of<float>(c, box.v, c->sigma1, c->rcut1, true, false);
    CU(launch_adj_gather<float>((const float4*)c->d_sorted, c->d_perm, n, sp, sg, c->p.ccelec,
                                gE_ch3, (const float*)c->d_rho, (const float*)c->d_phi, gd[0],
                                gd[1], gd[2], od[0], od[1], od[2], od[3], c->stream));
  }
  bool host = false;
  if (!dev_out) {
    double* outs[4] = {dq, dx, dy, dz};
    for (int k = 0; k < 4; k++) TRY(copy_out(c, outs[k], od[k], n * sizeof(double), &host));
  }
  return finish(c, host);
}

gse_status_t gse_ewald_recip(int device, void* stream, double sigma, int kcut, double box_x,
                             double box_y, double box_z, double ccelec, int n, const double* xyzq,
                             double* energy, double* fx, double* fy, double* fz) {
  g_last_error.clear();
  if (!(sigma > 0.0) || kcut < 1 || kcut > 255 || !(box_x > 0 && box_y > 0 && box_z > 0) ||
      n < 0 || (n > 0 && !xyzq) || !energy)
    return fail(GSE_ERR_INVALID_ARG, "bad Ewald arguments (kcut must lie in [1, 255])");
  const bool want_f = fx || fy || fz;
  if (want_f && !(fx && fy && fz)) return fail(GSE_ERR_INVALID_ARG, "give all force arrays or none");
  TRY(check_ptr(xyzq, device, sizeof(double4), "xyzq"));
  TRY(check_xyz(device, fx, fy, fz, "force array"));
  CU(cudaSetDevice(device));
  cudaStream_t st = (cudaStream_t)stream;
  const std::vector<EwRowHost> rows = ewald_rows(kcut);
  long long nk = 0;
  for (const EwRowHost& r : rows) nk += r.nk;
  EwGeom g;
  g.inv_box[0] = 1.0 / box_x;
  g.inv_box[1] = 1.0 / box_y;
  g.inv_box[2] = 1.0 / box_z;
  g.pref = 2.0 * kPi * g.inv_box[0] * g.inv_box[1] * g.inv_box[2] * ccelec;
  g.half_sigmasq = 0.5 * sigma * sigma;
  // scratch: rows, P S(k), row energies, and staged atoms/forces
  void* rows_d = nullptr;
  double2* S = nullptr;
  double* re = nullptr;
  double4* xd = nullptr;
  double* fd = nullptr;
  gse_status_t status = GSE_OK;
  std::vector<double> rh(rows.size());
  auto cleanup = [&]() {
    cudaFree(rows_d);
    cudaFree(S);
    cudaFree(re);
    cudaFree(xd);
    cudaFree(fd);
  };
#define CUE(call)                                                                          \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess) {                                                               \
      status = fail(_e == cudaErrorMemoryAllocation ? GSE_ERR_OOM : GSE_ERR_CUDA,          \
                    "gse_ewald_recip: %s: %s", #call, cudaGetErrorString(_e));             \
      cleanup();                                                                           \
      return status;                                                                       \
    }                                                                                      \
  } while (0)
  if (n == 0 || rows.empty()) {
    *energy = 0.0;
    return GSE_OK;
  }
  CUE(cudaMalloc(&rows_d, sizeof(EwRowHost) * rows.size()));
  CUE(cudaMalloc(&S, sizeof(double2) * nk));
  CUE(cudaMalloc(&re, sizeof(double) * rows.size()));
  const double4* xin = (const double4*)xyzq;
  if (!is_device_ptr(xyzq)) {
    CUE(cudaMalloc(&xd, sizeof(double4) * n));
    CUE(cudaMemcpyAsync(xd, xyzq, sizeof(double4) * n, cudaMemcpyHostToDevice, st));
    xin = xd;
  }
  double* f[3] = {fx, fy, fz};
  const bool fdev = want_f && is_device_ptr(fx) && is_device_ptr(fy) && is_device_ptr(fz);
  if (want_f && !fdev) {
    CUE(cudaMalloc(&fd, sizeof(double) * 3 * n));
    f[0] = fd;
    f[1] = fd + n;
    f[2] = fd + 2 * n;
  }
  EwScratch w{rows_d, S, re};
  CUE(launch_ewald(xin, n, rows, g, w, want_f ? f[0] : nullptr, f[1], f[2], st));
  CUE(cudaMemcpyAsync(rh.data(), re, sizeof(double) * rows.size(), cudaMemcpyDeviceToHost, st));
  if (want_f && !fdev) {
    CUE(cudaMemcpyAsync(fx, fd, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CUE(cudaMemcpyAsync(fy, fd + n, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CUE(cudaMemcpyAsync(fz, fd + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  }
  CUE(cudaStreamSynchronize(st));
#undef CUE
  double e = 0.0;
  for (double v : rh) e += v;
  *energy = e;
  cleanup();
  return GSE_OK;
}

gse_status_t gse_ewald_direct(int device, void* stream, double sigma, double rcut, double box_x,
                              double box_y, double box_z, double ccelec, int n, const double* xyzq,
                              int n_iblo14, const int* iblo14, const int* inb14, double* energy,
                              double* fx, double* fy, double* fz) {
  g_last_error.clear();
  if (!(sigma > 0.0) || !(rcut > 0.0) || !(box_x > 0 && box_y > 0 && box_z > 0) || n < 0 ||
      (n > 0 && !xyzq) || !energy || !std::isfinite(rcut) || !std::isfinite(sigma) ||
      !std::isfinite(box_x) || !std::isfinite(box_y) || !std::isfinite(box_z))
    return fail(GSE_ERR_INVALID_ARG, "bad Ewald direct arguments");
  const bool want_f = fx || fy || fz;
  if (want_f && !(fx && fy && fz)) return fail(GSE_ERR_INVALID_ARG, "give all force arrays or none");
  TRY(check_ptr(xyzq, device, sizeof(double4), "xyzq"));
  TRY(check_xyz(device, fx, fy, fz, "force array"));
  // exclusions: setupExclusions (CpuEwaldDirect.cpp:31-40) asks for one
  // cumulative end per atom (CpuEwaldDirect.cpp:47) and reads |inb14| - 1
  if (n_iblo14 < 0 || (n_iblo14 > 0 && (n_iblo14 != n || !iblo14)))
    return fail(GSE_ERR_INVALID_ARG, "iblo14 must hold one entry per atom");
  std::vector<int> ex_start, ex_idx;
  if (n_iblo14 > 0) {
    int prev = 0;
    for (int a = 0; a < n; a++) {
      if (iblo14[a] < prev)
        return fail(GSE_ERR_INVALID_ARG, "iblo14 must be non-decreasing from 0 (atom %d)", a);
      prev = iblo14[a];
    }
    if (prev > 0 && !inb14) return fail(GSE_ERR_INVALID_ARG, "inb14 is NULL");
    // the pair (a, b), a < b, is skipped when b is listed under a
    // (CpuEwaldDirect.cpp:71-85); entries at or below a never match
    std::vector<int> cnt(n + 1, 0);
    auto partner = [&](int k) { return (long long)std::llabs((long long)inb14[k]) - 1; };
    for (int a = 0, k = 0; a < n; a++)
      for (; k < iblo14[a]; k++) {
        const long long b = partner(k);
        if (b > a && b < n) {
          cnt[a]++;
          cnt[b]++;
        }
      }
    ex_start.assign(n + 1, 0);
    for (int a = 0; a < n; a++) ex_start[a + 1] = ex_start[a] + cnt[a];
    ex_idx.resize(ex_start[n]);
    std::vector<int> fill(ex_start.begin(), ex_start.end() - 1);
    for (int a = 0, k = 0; a < n; a++)
      for (; k < iblo14[a]; k++) {
        const long long b = partner(k);
        if (b > a && b < n) {
          ex_idx[fill[a]++] = (int)b;
          ex_idx[fill[b]++] = a;
        }
      }
    for (int a = 0; a < n; a++)
      std::sort(ex_idx.begin() + ex_start[a], ex_idx.begin() + ex_start[a + 1]);
  }
  CU(cudaSetDevice(device));
  cudaStream_t st = (cudaStream_t)stream;
  if (n == 0) {
    *energy = 0.0;
    return GSE_OK;
  }
  const double box[3] = {box_x, box_y, box_z};
  const EwdGeom g = ewald_direct_geom(sigma, rcut, box, ccelec);
  const int ntiles = (g.ncell + 4095) / 4096;
  // one allocation: ints, then doubles (8-byte aligned), then atoms
  const size_t n_int = 2 * (size_t)n + (size_t)g.ncell * 2 + 1 + ntiles + n + 1 + ex_idx.size() +
                       (ex_start.empty() ? 0 : n + 1);
  const size_t off_d = (n_int * sizeof(int) + 31) / 32 * 32;
  const size_t n_dbl = (size_t)g.ncell + 1 + (want_f ? 3 * (size_t)n : 0);
  const size_t off_x = (off_d + n_dbl * sizeof(double) + 31) / 32 * 32;
  const bool xdev = is_device_ptr(xyzq);
  const size_t bytes = off_x + (size_t)n * sizeof(double4) * (xdev ? 1 : 2);
  char* buf = nullptr;
  {
    cudaError_t e0 = cudaMalloc(&buf, bytes);
    if (e0 != cudaSuccess)
      return fail(e0 == cudaErrorMemoryAllocation ? GSE_ERR_OOM : GSE_ERR_CUDA,
                  "gse_ewald_direct: cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e0));
  }
  gse_status_t status = GSE_OK;
#define CUE(call)                                                                          \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess) {                                                               \
      status = fail(_e == cudaErrorMemoryAllocation ? GSE_ERR_OOM : GSE_ERR_CUDA,          \
                    "gse_ewald_direct: %s: %s", #call, cudaGetErrorString(_e));            \
      cudaFree(buf);                                                                       \
      return status;                                                                       \
    }                                                                                      \
  } while (0)
  int* ip = (int*)buf;
  EwdScratch w;
  w.key = ip;
  ip += n;
  w.tmp = ip;
  ip += n;
  w.counts = ip;
  ip += g.ncell;
  w.start = ip;
  ip += g.ncell + 1;
  w.tile_sums = ip;
  ip += ntiles;
  w.perm = ip;
  ip += n;
  w.done = (unsigned*)ip;
  ip += 1;
  int* d_ex_idx = ip;
  ip += ex_idx.size();
  int* d_ex_start = ex_start.empty() ? nullptr : ip;
  double* dp = (double*)(buf + off_d);
  w.partials = dp;
  double* d_energy = dp + g.ncell;
  double* f[3] = {fx, fy, fz};
  const bool fdev = want_f && is_device_ptr(fx) && is_device_ptr(fy) && is_device_ptr(fz);
  if (want_f && !fdev)
    for (int k = 0; k < 3; k++) f[k] = d_energy + 1 + (size_t)k * n;
  w.sorted = (double4*)(buf + off_x);
  const double4* xin = (const double4*)xyzq;
  if (!xdev) {
    double4* xd = w.sorted + n;
    CUE(cudaMemcpyAsync(xd, xyzq, sizeof(double4) * n, cudaMemcpyHostToDevice, st));
    xin = xd;
  }
  if (d_ex_start) {
    if (!ex_idx.empty())
      CUE(cudaMemcpyAsync(d_ex_idx, ex_idx.data(), sizeof(int) * ex_idx.size(),
                          cudaMemcpyHostToDevice, st));
    CUE(cudaMemcpyAsync(d_ex_start, ex_start.data(), sizeof(int) * (n + 1),
                        cudaMemcpyHostToDevice, st));
  }
  CUE(launch_ewald_direct(xin, n, g, w, d_ex_start, d_ex_start ? d_ex_idx : nullptr,
                          want_f ? f[0] : nullptr, f[1], f[2], d_energy, st));
  CUE(cudaMemcpyAsync(energy, d_energy, sizeof(double), cudaMemcpyDeviceToHost, st));
  if (want_f && !fdev) {
    CUE(cudaMemcpyAsync(fx, f[0], sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CUE(cudaMemcpyAsync(fy, f[1], sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CUE(cudaMemcpyAsync(fz, f[2], sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  }
  CUE(cudaStreamSynchronize(st));
#undef CUE
  cudaFree(buf);
  return GSE_OK;
}

}  // extern "C"
