// gse_ewald_direct.cu -- FP64 Ewald direct (real-space) sum on the GPU.
//
// CpuEwaldDirect::calcForceEnergy (CpuEwaldDirect.cpp:45-131): over the
// pairs (i, j) at minimum-image distance r < rcut that are not excluded,
//   E    = sum ccelec q_i q_j erfc(r / (sqrt2 sigma)) / r
//          - ccelec / sqrt(2 pi sigma^2) sum_i q_i^2,
//   f_ij = -ccelec q_i q_j (2 / sqrt(pi) / (sqrt2 sigma) exp(-r^2 / 2 sigma^2)
//          + erfc(r / (sqrt2 sigma)) / r) / r^2,
//   F_i  = sum_j f_ij (x_i - x_j)            (the gradient dE/dx_i).
// The pair (a, b), a < b, is excluded when b + 1 = |inb14[k]| for some k in
// [iblo14[a - 1], iblo14[a]) (CpuEwaldDirect.cpp:31-40, :71-85); the host
// turns those lists into one sorted list per atom holding both partners.
//
// Atoms are binned into cells of side >= rcut, stably (original order within
// a cell).  One CTA per cell takes the cell's atoms as i, 128 at a time, and
// streams the atoms of the neighbouring cells (the 3 nearest along an axis
// with at least 3 cells, every cell along a shorter one) through shared
// memory as j.  Every pair term is formed by both partners' threads, so each
// atom's force and half of its pair energies are summed by one thread in a
// fixed order: the results do not depend on scheduling.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>

#include "gse_ewald.cuh"
#include "gse_internal.cuh"
#include "gse_reduce.cuh"
#include "gse_tiled.cuh"

namespace gse {

constexpr int kEwdThreads = 128;

// Cell index of a coordinate along one axis: the position taken into
// [0, box) and scaled by nc / box, clamped to [0, nc).
__device__ __forceinline__ int ewd_cell_axis(double x, double box, double inv_box, int nc) {
  const double w = x - box * floor(x * inv_box);
  const int c = (int)(w * inv_box * (double)nc);
  return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__global__ void k_ewd_cell_count(const double4* __restrict__ xyzq, int n, EwdGeom g,
                                 int* __restrict__ key, int* __restrict__ counts) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double4 p = xyzq[i];
    const int cx = ewd_cell_axis(p.x, g.box[0], g.inv_box[0], g.nc[0]);
    const int cy = ewd_cell_axis(p.y, g.box[1], g.inv_box[1], g.nc[1]);
    const int cz = ewd_cell_axis(p.z, g.box[2], g.inv_box[2], g.nc[2]);
    const int k = cx + g.nc[0] * (cy + g.nc[1] * cz);
    key[i] = k;
    atomicAdd(&counts[k], 1);
  }
}

// The minimum image of d as the reference's while loops leave it: within
// [-box/2, box/2], a difference of exactly +-box/2 kept as it is.
__device__ __forceinline__ double ewd_min_image(double d, double box, double hbox,
                                                double inv_box) {
  if (d < -hbox || d > hbox) {
    d -= box * rint(d * inv_box);
    if (d < -hbox) d += box;
    if (d > hbox) d -= box;
  }
  return d;
}

__global__ void __launch_bounds__(kEwdThreads)
    k_ewd_pairs(const double4* __restrict__ sorted, const int* __restrict__ perm,
                const int* __restrict__ start, EwdGeom g, const int* __restrict__ ex_start,
                const int* __restrict__ ex_idx, double* __restrict__ fx, double* __restrict__ fy,
                double* __restrict__ fz, double* __restrict__ partials, unsigned* done,
                double* __restrict__ energy_out) {
  __shared__ double4 sj[kEwdThreads];
  __shared__ int sid[kEwdThreads];
  const int tid = threadIdx.x;
  const int cell = blockIdx.x;
  const int c[3] = {cell % g.nc[0], (cell / g.nc[0]) % g.nc[1], cell / (g.nc[0] * g.nc[1])};
  int lo[3], cnt[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    lo[d] = g.nc[d] >= 3 ? c[d] - 1 + g.nc[d] : 0;
    cnt[d] = g.nc[d] >= 3 ? 3 : g.nc[d];
  }
  const int i0 = start[cell], i1 = start[cell + 1];
  double esum = 0.0;
  for (int ib = i0; ib < i1; ib += kEwdThreads) {  // uniform in the CTA
    const int i = ib + tid;
    const bool act = i < i1;
    const double4 pi = act ? sorted[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    const int oi = act ? perm[i] : -1;
    int e0 = 0, e1 = 0;
    if (act && ex_start) {
      e0 = ex_start[oi];
      e1 = ex_start[oi + 1];
    }
    const double qi = g.ccelec * pi.w;
    double fxa = 0.0, fya = 0.0, fza = 0.0, ea = 0.0;
    for (int oz = 0; oz < cnt[2]; oz++)
      for (int oy = 0; oy < cnt[1]; oy++)
        for (int ox = 0; ox < cnt[0]; ox++) {
          const int nb = (lo[0] + ox) % g.nc[0] +
                         g.nc[0] * ((lo[1] + oy) % g.nc[1] + g.nc[1] * ((lo[2] + oz) % g.nc[2]));
          const int j0 = start[nb], j1 = start[nb + 1];
          for (int jb = j0; jb < j1; jb += kEwdThreads) {
            __syncthreads();  // the previous tile is consumed
            if (jb + tid < j1) {
              sj[tid] = sorted[jb + tid];
              sid[tid] = perm[jb + tid];
            }
            __syncthreads();
            const int m = min(kEwdThreads, j1 - jb);
            if (!act) continue;
            for (int k = 0; k < m; k++) {
              const double4 pj = sj[k];
              const double dx = ewd_min_image(pi.x - pj.x, g.box[0], g.hbox[0], g.inv_box[0]);
              const double dy = ewd_min_image(pi.y - pj.y, g.box[1], g.hbox[1], g.inv_box[1]);
              const double dz = ewd_min_image(pi.z - pj.z, g.box[2], g.hbox[2], g.inv_box[2]);
              const double r2 = dx * dx + dy * dy + dz * dz;
              if (!(r2 < g.rcut2)) continue;
              const int oj = sid[k];
              if (oj == oi) continue;
              bool excl = false;
              for (int e = e0; e < e1; e++) excl |= ex_idx[e] == oj;
              if (excl) continue;
              const double qq = qi * pj.w;
              const double r = sqrt(r2);
              const double erfcval = erfc(r * g.inv_sqrt2sigma);
              const double expval = exp(-r2 * g.inv_2sigmasq);
              const double f = -qq * (g.two_sqrtpi * g.inv_sqrt2sigma * expval + erfcval / r) / r2;
              fxa += f * dx;
              fya += f * dy;
              fza += f * dz;
              ea += qq * erfcval / r;
            }
          }
        }
    if (act) {
      if (fx) {
        fx[oi] = fxa;
        fy[oi] = fya;
        fz[oi] = fza;
      }
      esum += 0.5 * ea + g.self * pi.w * pi.w;
    }
  }
  block_sum_to(esum, partials);
  last_block_sum_counter(partials, done, 1.0, energy_out);
}

EwdGeom ewald_direct_geom(double sigma, double rcut, const double box[3], double ccelec) {
  EwdGeom g;
  long long cells = 1;
  for (int d = 0; d < 3; d++) {
    g.box[d] = box[d];
    g.hbox[d] = 0.5 * box[d];
    g.inv_box[d] = 1.0 / box[d];
    // a relative margin keeps the side >= rcut through the rounding of the
    // cell index
    const double q = box[d] / (rcut * (1.0 + 1e-9));
    g.nc[d] = q >= (double)kEwdMaxCellsPerAxis ? kEwdMaxCellsPerAxis : (q < 1.0 ? 1 : (int)q);
    cells *= g.nc[d];
  }
  g.ncell = (int)cells;
  g.rcut2 = rcut * rcut;
  g.inv_sqrt2sigma = 1.0 / (std::sqrt(2.0) * sigma);
  g.inv_2sigmasq = 1.0 / (2.0 * sigma * sigma);
  g.two_sqrtpi = 2.0 / std::sqrt(kPi);
  g.self = -ccelec / std::sqrt(2.0 * kPi * sigma * sigma);
  g.ccelec = ccelec;
  return g;
}

cudaError_t launch_ewald_direct(const double4* xyzq, int n, const EwdGeom& g, EwdScratch w,
                                const int* ex_start, const int* ex_idx, double* fx, double* fy,
                                double* fz, double* energy_out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(w.counts, 0, sizeof(int) * g.ncell, st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(w.done, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  const int gb = n > 0 ? (int)std::min<long long>(sm_count() * 8, (n + 255) / 256) : 1;
  if (n > 0) k_ewd_cell_count<<<gb, 256, 0, st>>>(xyzq, n, g, w.key, w.counts);
  BinScratch b;
  b.key = w.key;
  b.counts = w.counts;
  b.start = w.start;
  b.tile_sums = w.tile_sums;
  b.tmp = w.tmp;
  b.qmax_bits = nullptr;
  e = launch_bin_scan_place<double>(xyzq, n, g.ncell, b, w.sorted, w.perm, st);
  if (e != cudaSuccess) return e;
  k_ewd_pairs<<<g.ncell, kEwdThreads, 0, st>>>(w.sorted, w.perm, w.start, g, ex_start, ex_idx,
                                               fx, fy, fz, w.partials, w.done, energy_out);
  return cudaGetLastError();
}

}  // namespace gse
