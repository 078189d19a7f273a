// gse_tiled.cuh -- tiled spread / gather kernels and the atom binning they use.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "gse_internal.cuh"

namespace gse {

// x cells per bin (y and z bins are single cells): the FP64 spread reads atom
// ranges at 4-cell granularity; every mixed-form kernel reads whole 16-cell
// brick rows, so the mixed form bins 16 cells at a time (4x fewer bins to scan)
constexpr int kBinX64 = 4, kBinX32 = 16;
constexpr int kWPad = 16;           // padded stencil width (2n+1 <= 15 on the tiled path)
constexpr int kTX = 16, kTY = 8;    // spread block columns (x, y)
constexpr int kTZ32 = 32;           // spread block depth, mixed form (int64 accumulators)
constexpr int kTZ64 = 24;           // spread block depth, FP64 accumulators
constexpr int kSpreadThreads = 128; // 4 warps, each an 8 x 4 column patch
constexpr int kSpreadChunk = 64;    // atoms staged per round
constexpr int kMaxSeg = 4;          // periodic images of one row segment
constexpr int kGX = 16, kGY = 16, kGZ = 8;  // gather brick (cells); kGX multiple of kBinX32
constexpr int kGatherThreads = 256;          // >= kGY * kGZ
constexpr int kGatherLanes = 16;             // lanes sharing one atom in the gather
constexpr int kMinTiledGrid = 10;   // smallest grid side on the tiled path
constexpr int kSB = 16;             // scatter-spread brick (cells per axis)
constexpr int kFlushBits = 40;  // scale of the int64 accumulation grids
constexpr int kScatterThreads = 512;  // >= kSB * kSB
constexpr int kScatterList = 1024;  // atoms per scatter round (per brick)
constexpr int kGatherList = 512;    // atoms per gather round (per brick)
constexpr int kAX = 16, kAY = 8, kAZ = 8;  // reverse-pass gather brick (two staged grids)
constexpr int kAdjThreads = 256;           // >= kAY * kAZ
// lanes per atom in the reverse-pass gather: a whole warp (two atoms per warp
// would need more shared memory than two blocks per SM leave for its tables)
constexpr int kAdjLanes = 32;

// Atoms sorted by key (z cell, y cell, x bin); start[k] .. start[k+1] is bin k.
struct BinLayout {
  int M[3];
  int nbx;    // ceil(Mx / bin width)
  int bxs;    // log2 of the bin width in x cells
  // mixed-form scatter: set to kFlagRange when a brick's charge exceeds the
  // fixed-point range of its int32 tile (may be NULL: not reported)
  int* flags = nullptr;
};

struct BinScratch {
  int* key;        // [n]
  int* counts;     // [nbins]
  int* start;      // [nbins + 1]
  int* tile_sums;  // [ceil(nbins / 4096)]
  int* tmp;        // [n]: the FP64 stable placement's scratch; the mixed form's ranks in bin
  unsigned* qmax_bits;  // max |q| over the atoms (float bits), written by the binning
  int* bad = nullptr;   // set to 1 when a position or charge is not finite (may be NULL)
  // mixed form: the scan's tile-local prefix [nbins] (the placement applies the tile
  // offsets and writes `start`); NULL: a three-kernel scan writes `start` directly
  int* lstart = nullptr;
  // mixed form: `counts` are zero on entry (the order-free placement counts every
  // bin back down to zero), so the binning does not clear them
  bool counts_zero = false;
  // an int64 array of clear_n elements (16-byte aligned) that the counting
  // kernel clears on the way (the mixed form's spread grid); NULL: none
  long long* clear = nullptr;
  long long clear_n = 0;
};

// exp(-2 h^2 / (2 sigma^2)) per axis as an unevaluated sum hi + lo in CT
template <typename CT>
struct Decay {
  CT hi[3], lo[3];
};
template <typename CT>
inline Decay<CT> make_decay(const Stencil<CT>& s) {
  Decay<CT> d;
  for (int a = 0; a < 3; a++) {
    const double hd = (double)s.h[a];
    const double v = std::exp(-2.0 * hd * hd * (double)s.inv_2s2);
    d.hi[a] = (CT)v;
    d.lo[a] = (CT)(v - (double)d.hi[a]);
  }
  return d;
}

inline BinLayout make_bin_layout(const int M[3], int bin_width) {
  BinLayout b;
  for (int d = 0; d < 3; d++) b.M[d] = M[d];
  b.bxs = bin_width == 16 ? 4 : 2;
  b.nbx = (M[0] + (1 << b.bxs) - 1) >> b.bxs;
  return b;
}
static_assert(kGX % kBinX32 == 0 && kSB % kBinX32 == 0 && kAX % kBinX32 == 0,
              "mixed-form bricks start on bin boundaries");

inline int bin_count(const BinLayout& b) { return b.M[1] * b.M[2] * b.nbx; }

// One system of a batch (mixed form).  Atoms of all systems are binned with
// one global key: bin_off + the system's own (z cell, y cell, x bin) key.
struct BatchSys {
  BinLayout b;
  int bin_off;          // first bin of the system
  int atom_off, n;      // atom range in the caller's concatenated order
  int W;                // stencil width 2n+1
  long long grid_off;   // first point of the system's real grids
  long long kgrid_off;  // first bin of its half spectrum
  double efac;          // 1/2 ccelec hx hy hz
  double h3;            // hx hy hz
  Stencil<float> sp;    // spread stencil (sigma1, rcut1)
  Stencil<float> sg;    // gather stencil
};

struct BatchItem {
  int sys, bx, by, bz;  // brick of one system
};

// A run of work items whose systems share one stencil width W (the batched
// kernels are instantiated per width; one launch per run).
struct BatchSeg {
  int W, first, count;
};

// The batched evaluation in one persistent cooperative launch per direction:
// binning, spread, the small-grid FFT solve with the Green's multiply and
// energy, and gather (forward), or adjoint source, solve and reverse-pass
// gather (reverse), separated by grid-wide barriers.  Grids must be multiples
// of 8 and at most 64 points per side (batch_fused_supported).
struct BatchFused {
  const float4* xyzq;
  int ntot, nsys, nbins;
  const BatchSys* sys;
  const int* first;         // [nsys + 1] first atom of each system
  BinScratch w;
  float4* sorted;
  int* perm;
  const BatchItem* scat;    // spread / adjoint-source bricks
  int nscat;
  const BatchItem* gath;    // gather bricks
  int ngath;
  const BatchItem* agath;   // reverse-pass gather bricks
  int nagath;
  long long* g64;           // int64 accumulation grid (all systems)
  long long gtot;
  float2* rhok;             // half spectra
  const float* gtab;        // Green's tables (half-spectrum layout)
  float* phi;               // potential
  float* psi;               // reverse-pass potential of the adjoint source
  const int* xrow_first;    // [nsys + 1] prefix of the systems' x rows (My Mz)
  const int* ycol_first;    // [nsys + 1] prefix of their y columns (Mz (Mx/2+1))
  const int* zcol_first;    // [nsys + 1] prefix of their z columns (My (Mx/2+1))
  double* epart;            // [zcol_first[nsys]] k-space energy of each z column
  double* energy;           // [nsys]
  double ccelec;
  double *fx, *fy, *fz;     // forces [ntot]
  const double* dLdE;       // reverse pass inputs
  const double *gfx, *gfy, *gfz;
  double *dq, *dx, *dy, *dz;  // reverse pass outputs
  int* qctr;                // [4] work-item counters: spread, gather, adjoint source,
                            // reverse-pass gather (each kernel zeroes its own first)
};

bool batch_fused_supported(const BatchSys* sys, int nsys);
// Largest cooperative grid of the fused kernels on this device (0: cannot run).
int batch_fused_ctas(int gather_lanes);
int batch_fused_rev_ctas();
cudaError_t launch_batch_forward_fused(const BatchFused& a, int ctas, int gather_lanes,
                                       cudaStream_t st);
cudaError_t launch_batch_reverse_fused(const BatchFused& a, int ctas, cudaStream_t st);

cudaError_t launch_batch_bin(const float4* xyzq, int ntot, const BatchSys* sys, const int* first,
                             int nsys, int nbins, BinScratch w, float4* sorted, int* perm,
                             cudaStream_t st);
cudaError_t launch_batch_spread(const float4* sorted, const int* start, const BatchSys* sys,
                                const BatchItem* items, const BatchSeg* segs, int nseg, int ctas,
                                long long* grid64, long long gsize, float* rho, cudaStream_t st);
cudaError_t launch_batch_green(float2* rhok, const float* tab, long long ktot, const BatchSys* sys,
                               const long long* kfirst, const int* ksys, int nsys, double* energy,
                               cudaStream_t st);
cudaError_t launch_batch_gather(const float4* sorted, const int* perm, const int* start,
                                const BatchSys* sys, const BatchItem* items, const BatchSeg* segs,
                                int nseg, int ctas, const float* phi, double outscale, double* fx,
                                double* fy, double* fz, cudaStream_t st);

// float grid = int64 accumulation grid at 2^40 (the scatter kernels' output)
cudaError_t launch_grid64_to_real(const long long* grid64, long long size, float* out,
                                  cudaStream_t st);

// Mixed-form spread: brick tiles added into the int64 grid `grid64` at 2^40,
// then converted into the float grid `rho` (NULL: left to the caller).  The
// grid is cleared here unless `zeroed`: the caller cleared it before the
// binning, and the spread then launches as the dependent of the binning's
// last kernel, which directly precedes it on `st`.
cudaError_t launch_spread_scatter(const float4* sorted, const int* start, const BinLayout& b,
                                  const Stencil<float>& s, long long* grid64, float* rho,
                                  bool zeroed, cudaStream_t st);

template <typename CT>
cudaError_t launch_bin_sorted(const typename Vec4<CT>::type* xyzq, int n, const BinLayout& b,
                              CT inv_hx, CT inv_hy, CT inv_hz, BinScratch w,
                              typename Vec4<CT>::type* sorted, int* perm, cudaStream_t st);

template <typename CT>
cudaError_t launch_bin_scan_place(const typename Vec4<CT>::type* xyzq, int n, int nb,
                                  BinScratch w, typename Vec4<CT>::type* sorted, int* perm,
                                  cudaStream_t st);

template <typename CT>
bool spread_tiled_supported(const Stencil<CT>& s);

template <typename CT>
cudaError_t launch_spread_tiled(const typename Vec4<CT>::type* sorted, const int* start,
                                const unsigned* qmax_bits, const BinLayout& b,
                                const Stencil<CT>& s, CT* grid, cudaStream_t st);

// pdl: the launch follows a kernel of this library directly on `st` and may
// overlap its end (programmatic dependent launch).
template <typename CT>
cudaError_t launch_gather_tiled(const typename Vec4<CT>::type* sorted, const int* perm,
                                const int* start, const BinLayout& b, const Stencil<CT>& s,
                                const CT* phi, double outscale, double* fx, double* fy,
                                double* fz, bool pdl, cudaStream_t st);

}  // namespace gse
