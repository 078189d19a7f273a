// gse_tiled_dev.cuh -- device helpers shared by the tiled forward kernels
// (gse_tiled.cu) and the tiled reverse-pass kernels (gse_adjoint.cu).
#pragma once

#include <cooperative_groups.h>

#include "gse_internal.cuh"
#include "gse_smallfft.cuh"
#include "gse_tiled.cuh"

namespace gse {

// Grid cell nearest to a coordinate (the stencil centre), not yet wrapped.
template <typename CT>
__device__ __forceinline__ int centre_cell(CT v, CT inv_h) {
  return round_to_int(mul_rn(v, inv_h));
}

// Exclusive prefix sum of one int per thread over the whole block; *total
// receives the block's sum.  All threads of the block must call it.
__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
  __shared__ int ws[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    int s = (lane < nw) ? ws[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    ws[lane] = s;
  }
  __syncthreads();
  const int before = (w > 0 ? ws[w - 1] : 0) + x - v;
  if (total) *total = ws[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before;
}

// ---------------------------------------------------------------------------
// Brick tiles of the scatter kernels (forward spread and adjoint source).
// ---------------------------------------------------------------------------
// Shared int32 tile of one kSB^3 brick plus its n-point halo, T points per
// axis; the z-plane pitch is congruent to 2n+1 mod 32 so that the 32 lanes of
// one instruction (consecutive (x, z) pairs of a stencil plane) hit 32
// different banks.
template <int W>
struct ScatterGeom {
  static constexpr int n = (W - 1) / 2;
  static constexpr int T = kSB + 2 * n;
  static constexpr int RP = T;                              // y pitch
  static constexpr int PP = ((T * T + 31) / 32) * 32 + W;   // z pitch, = W (mod 32)
  static constexpr int words = T * PP;
};

constexpr int kMinShift = 11;   // 2^30 * 2^(40-11) * 8 overlapping tiles < 2^63

// Block prologue of a scatter brick: the brick's atoms (one contiguous range
// per (y, z) cell row, start offsets in rng_a, exclusive prefix in rng_p),
// the cleared tile, and the brick's power-of-two scale 2^S such that the sum
// of bound(i) over its atoms times 2^S stays below 2^30 and every single
// bound(i) times 2^S below 2^22.  bound(i) is an upper bound of |contribution|
// of sorted atom i to any one grid point.  Returns S; *total gets the atom
// count.  All threads of the block must call it.
template <int W, int NT, class Bound>
__device__ __forceinline__ int brick_prologue(const int* __restrict__ start, const BinLayout& b,
                                              int x0, int y0, int z0, int* __restrict__ tile,
                                              int* rng_a, int* rng_p, Bound bound, int* total) {
  typedef ScatterGeom<W> G;
  constexpr int NW = NT / 32;
  __shared__ double qsum_w[NW];
  __shared__ float qmax_w[NW];
  __shared__ int s_shift;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ex = min(kSB, b.M[0] - x0), ey = min(kSB, b.M[1] - y0), ez = min(kSB, b.M[2] - z0);
  int cnt = 0, a0 = 0;
  if (tid < kSB * kSB) {
    const int yy = tid % kSB, zz = tid / kSB;
    if (yy < ey && zz < ez) {
      const int rowkey = ((z0 + zz) * b.M[1] + (y0 + yy)) * b.nbx;
      a0 = start[rowkey + (x0 >> b.bxs)];
      cnt = start[rowkey + ((x0 + ex - 1) >> b.bxs) + 1] - a0;
    }
  }
  const int pos = block_exclusive_scan(cnt, total);
  if (tid < kSB * kSB) {
    rng_a[tid] = a0;
    rng_p[tid] = pos;
  }
  for (int i = tid; i < G::words / 4; i += NT)
    reinterpret_cast<int4*>(tile)[i] = make_int4(0, 0, 0, 0);
  for (int i = (G::words / 4) * 4 + tid; i < G::words; i += NT) tile[i] = 0;
  // double sums of the float bounds: exact for any realistic spread of
  // magnitudes, so the scale does not depend on the order of a bin's atoms
  double qs = 0.0;
  float qm = 0.f;
  for (int j = 0; j < cnt; j++) {
    const float q = bound(a0 + j);
    qs += (double)q;
    qm = fmaxf(qm, q);
  }
  qs = warp_sum(qs);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) qm = fmaxf(qm, __shfl_xor_sync(0xffffffffu, qm, o));
  if (lane == 0) {
    qsum_w[warp] = qs;
    qmax_w[warp] = qm;
  }
  __syncthreads();
  if (tid == 0) {
    double q = 0.0;
    float m = 0.f;
    for (int w = 0; w < NW; w++) {
      q += qsum_w[w];
      m = fmaxf(m, qmax_w[w]);
    }
    const double sum_b = q * 1.0001 + 1e-30;
    const double one_b = (double)m * 1.0001 + 1e-30;
    int sh = kFlushBits;
    while (sh > kMinShift && (sum_b * exp2((double)sh) >= 1073741824.0 ||
                              one_b * exp2((double)sh) >= 4194304.0))
      sh--;
    // even the coarsest scale leaves the tile's int32 sums without headroom:
    // the brick's result would wrap, so the call reports a range error
    // (non-finite charges are the binning's report)
    if ((sum_b * exp2((double)sh) >= 1073741824.0 || one_b * exp2((double)sh) >= 4194304.0) &&
        isfinite(sum_b) && b.flags)
      *b.flags = kFlagRange;
    s_shift = sh;
  }
  __syncthreads();
  return s_shift;
}

// Flat list alist[0 .. min(chunk, total - c0)) of the brick's atoms c0, c0+1,
// ... (block-wide; the caller synchronises before reading it).
template <int NT, int NROWS>
__device__ __forceinline__ void brick_atom_list(const int* rng_a, const int* rng_p, int total,
                                                int c0, int chunk, int* alist) {
  for (int r = threadIdx.x; r < NROWS; r += NT) {
    const int p0 = rng_p[r];
    const int p1 = (r + 1 < NROWS) ? rng_p[r + 1] : total;
    for (int p = max(p0, c0); p < min(p1, c0 + chunk); p++) alist[p - c0] = rng_a[r] + (p - p0);
  }
}

// Finished tile (values at 2^shift) -> int64 grid at 2^kFlushBits (shift <=
// kFlushBits, so the scaling is exact) by integer reductions, which do not
// depend on their order.
template <int W, int NT>
__device__ __forceinline__ void brick_flush(const int* __restrict__ tile, const BinLayout& b,
                                            int x0, int y0, int z0, int shift,
                                            long long* __restrict__ grid64) {
  typedef ScatterGeom<W> G;
  constexpr int n = G::n, T = G::T;
  static_assert(T <= 32, "one lane per tile column");
  const long long mul = 1LL << (kFlushBits - shift);
  // one lane per x (its wrapped x is the same everywhere); warp w takes the
  // tile rows y = w, w + NT/32, ..., and walks each row's z column with the
  // global plane advanced by one step (wrapping at M[2]), so the index
  // arithmetic per element is one step, not a wrap per axis
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane >= T) return;
  const long long zs = (long long)b.M[0] * b.M[1];
  unsigned long long* gxp = (unsigned long long*)grid64 + wrap1(x0 - n + lane, b.M[0]);
  const int gz0 = wrap1(z0 - n, b.M[2]);
  for (int yy = warp; yy < T; yy += NT / 32) {
    unsigned long long* gyp = gxp + (long long)wrap1(y0 - n + yy, b.M[1]) * b.M[0];
    const int* t = tile + yy * T + lane;
    int gz = gz0;
#pragma unroll 4
    for (int zz = 0; zz < T; zz++) {
      const int v = t[zz * G::PP];
      if (v != 0) atomicAdd(gyp + gz * zs, (unsigned long long)((long long)v * mul));
      gz = (gz + 1 == b.M[2]) ? 0 : gz + 1;
    }
  }
}

// Stage the potential-like grid `src` for a brick at (x0, y0, z0) with an
// n-point halo into the shared tile [TZ][ZP] (rows of pitch TP) by
// asynchronous element copies; the caller waits (cp.async.wait_all) and
// synchronises.
template <typename CT, int TX, int TY, int TZ, int TP, int ZP, int NW>
__device__ __forceinline__ void stage_tile_async(const CT* __restrict__ src, const BinLayout& b,
                                                 int x0, int y0, int z0, int n, CT* tile) {
  static_assert(TX <= 32, "one lane per tile column");
  // one lane per x (its wrapped x is the same everywhere); warp w takes the
  // tile rows y = w, w + NW, ..., and walks each row's z column with the
  // global plane advanced by one step (wrapping at M[2])
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane >= TX) return;
  const long long zs = (long long)b.M[0] * b.M[1];
  const CT* sx = src + wrap1(x0 - n + lane, b.M[0]);
  const int gz0 = wrap1(z0 - n, b.M[2]);
  const unsigned base = (unsigned)__cvta_generic_to_shared(tile + lane);
  for (int ty = warp; ty < TY; ty += NW) {
    const CT* sy = sx + (long long)wrap1(y0 - n + ty, b.M[1]) * b.M[0];
    unsigned dst = base + (unsigned)(ty * TP * sizeof(CT));
    int gz = gz0;
#pragma unroll 4
    for (int tz = 0; tz < TZ; tz++) {
      asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(dst), "l"(sy + gz * zs),
                   "n"(sizeof(CT))
                   : "memory");
      dst += (unsigned)(ZP * sizeof(CT));
      gz = (gz + 1 == b.M[2]) ? 0 : gz + 1;
    }
  }
}

// ---------------------------------------------------------------------------
// Batched systems
// ---------------------------------------------------------------------------
// Next work item of a phase for the whole block, from a counter in global
// memory: blocks take items as they finish the previous one, so a phase ends
// with the blocks' loads balanced.  All threads of the block must call it.
__device__ __forceinline__ int fused_next_item(int* ctr) {
  __shared__ int next;
  __syncthreads();
  if (threadIdx.x == 0) next = atomicAdd(ctr, 1);
  __syncthreads();
  return next;
}

// System of item i, given each system's first item in first[0..nsys).
__device__ __forceinline__ int batch_sys_of(const int* __restrict__ first, int nsys, int i) {
  int lo = 0, hi = nsys - 1;  // last s with first[s] <= i
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// The small-grid FFT solve of every system (forward: from the int64 spread
// grid to the potential, with the k-space energy; reverse: the adjoint source
// to its potential, no energy): five passes of independent lines, one group of
// 8 lanes per line (gse_smallfft.cuh), separated by grid-wide barriers.  All
// threads of the cooperative grid call it.
struct SfLine {
  int s, r;     // system, line index within the system's pass
  bool active;  // false for the padding groups past the last line
};

// Largest system count whose line prefixes the FFT passes stage in shared memory.
constexpr int kSfSmemSystems = 2047;

__device__ __forceinline__ SfLine sf_line(const int* first, int nsys, int u) {
  SfLine L;
  L.active = u < first[nsys];
  L.s = L.active ? batch_sys_of(first, nsys, u) : 0;
  L.r = L.active ? u - first[L.s] : 0;
  return L;
}

// Group loop over the lines of one pass: every warp of the grid takes eight
// consecutive lines at a time, two per group (u0 and u1 = u0 + 4), so all its
// lanes run the shuffles together and each group has two independent lines in
// flight.
#define SF_FOR_LINE_PAIRS(total, u0, u1)                                                \
  for (int sf_w0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 8;                  \
       sf_w0 < (total); sf_w0 += (gridDim.x * blockDim.x) >> 2)                         \
    for (int u0 = sf_w0 + ((threadIdx.x & 31) >> 3), u1 = u0 + 4, sf_once = 1; sf_once;  \
         sf_once = 0)

__device__ __forceinline__ void fused_solve(const BatchFused& a, float* out, bool energy,
                                            unsigned char* fsm) {
  namespace cg = cooperative_groups;
  SmallFftTw& T = *reinterpret_cast<SmallFftTw*>(fsm);
  sf_build_twiddles(T);
  // the passes' line prefixes in shared memory: every line looks up its system
  // by a binary search over them
  const int* xrow_first = a.xrow_first;
  const int* ycol_first = a.ycol_first;
  const int* zcol_first = a.zcol_first;
  if (a.nsys <= kSfSmemSystems) {
    int* pre = reinterpret_cast<int*>(fsm + sizeof(SmallFftTw));
    const int np = a.nsys + 1;
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
      pre[i] = a.xrow_first[i];
      pre[np + i] = a.ycol_first[i];
      pre[2 * np + i] = a.zcol_first[i];
    }
    xrow_first = pre;
    ycol_first = pre + np;
    zcol_first = pre + 2 * np;
  }
  __syncthreads();
  const int l = threadIdx.x & 7, k1 = bitrev3(l);
  const double unscale = exp2(-40.0);
  // x rows: r2c of the int64 grid
  SF_FOR_LINE_PAIRS(xrow_first[a.nsys], u0, u1) {
    SfLine L[2] = {sf_line(xrow_first, a.nsys, u0), sf_line(xrow_first, a.nsys, u1)};
    float2 v[2][8];
    int m[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const BatchSys& S = a.sys[L[q].s];
      const int Mx = S.b.M[0];
      m[q] = L[q].active ? Mx / 8 : 1;
      const long long* g = a.g64 + S.grid_off + (long long)L[q].r * Mx;
#pragma unroll
      for (int j1 = 0; j1 < 8; j1++)
        v[q][j1] = (L[q].active && j1 < m[q])
                       ? make_float2((float)((double)g[m[q] * l + j1] * unscale), 0.f)
                       : make_float2(0.f, 0.f);
    }
    const int mmax = sf_warp_mmax(max(m[0], m[1]));
    sf8_dft(v[0], m[0], mmax, -1.f, T);
    sf8_dft(v[1], m[1], mmax, -1.f, T);
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const BatchSys& S = a.sys[L[q].s];
      const int Hx = S.b.M[0] / 2 + 1;
      float2* o = a.rhok + S.kgrid_off + (long long)L[q].r * Hx;
#pragma unroll
      for (int k2 = 0; k2 < 8; k2++)
        if (L[q].active && k2 < m[q] && k1 + 8 * k2 < Hx) o[k1 + 8 * k2] = v[q][k2];
    }
  }
  cg::this_grid().sync();
  // y columns, forward then (after the z pass) inverse
  auto ypass = [&](float dir) {
    SF_FOR_LINE_PAIRS(ycol_first[a.nsys], u0, u1) {
      SfLine L[2] = {sf_line(ycol_first, a.nsys, u0), sf_line(ycol_first, a.nsys, u1)};
      float2 v[2][8];
      float2* c[2];
      int m[2];
      long long hx[2];
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const BatchSys& S = a.sys[L[q].s];
        const int Hx = S.b.M[0] / 2 + 1, My = S.b.M[1];
        m[q] = L[q].active ? My / 8 : 1;
        hx[q] = Hx;
        const int z = L[q].r / Hx, x = L[q].r - z * Hx;
        c[q] = a.rhok + S.kgrid_off + (long long)z * My * Hx + x;
#pragma unroll
        for (int j1 = 0; j1 < 8; j1++)
          v[q][j1] = (L[q].active && j1 < m[q]) ? c[q][(m[q] * l + j1) * hx[q]]
                                                : make_float2(0.f, 0.f);
      }
      const int mmax = sf_warp_mmax(max(m[0], m[1]));
      sf8_dft(v[0], m[0], mmax, dir, T);
      sf8_dft(v[1], m[1], mmax, dir, T);
#pragma unroll
      for (int q = 0; q < 2; q++)
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++)
          if (L[q].active && k2 < m[q]) c[q][(k1 + 8 * k2) * hx[q]] = v[q][k2];
    }
  };
  ypass(-1.f);
  cg::this_grid().sync();
  // z columns: forward, Green's multiply (and energy), inverse
  SF_FOR_LINE_PAIRS(zcol_first[a.nsys], u0, u1) {
    SfLine L[2] = {sf_line(zcol_first, a.nsys, u0), sf_line(zcol_first, a.nsys, u1)};
    float2 v[2][8];
    float2* c[2];
    const float* gt[2];
    long long pitch[2];
    int m[2];
    double wgt[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const BatchSys& S = a.sys[L[q].s];
      const int Mx = S.b.M[0], Hx = Mx / 2 + 1, My = S.b.M[1], Mz = S.b.M[2];
      m[q] = L[q].active ? Mz / 8 : 1;
      const int y = L[q].r / Hx, x = L[q].r - y * Hx;
      pitch[q] = (long long)My * Hx;
      const long long off = S.kgrid_off + (long long)y * Hx + x;
      c[q] = a.rhok + off;
      gt[q] = a.gtab + off;
      wgt[q] = (x == 0 || x == Mx / 2) ? 1.0 : 2.0;
#pragma unroll
      for (int j1 = 0; j1 < 8; j1++)
        v[q][j1] = (L[q].active && j1 < m[q]) ? c[q][(m[q] * l + j1) * pitch[q]]
                                              : make_float2(0.f, 0.f);
    }
    const int mmax = sf_warp_mmax(max(m[0], m[1]));
    sf8_dft(v[0], m[0], mmax, -1.f, T);
    sf8_dft(v[1], m[1], mmax, -1.f, T);
    double e[2] = {0.0, 0.0};
#pragma unroll
    for (int q = 0; q < 2; q++)
#pragma unroll
      for (int k2 = 0; k2 < 8; k2++) {
        if (L[q].active && k2 < m[q]) {
          const float f = gt[q][(k1 + 8 * k2) * pitch[q]];
          const float2 w = v[q][k2];
          if (energy) e[q] += wgt[q] * (double)f * ((double)w.x * w.x + (double)w.y * w.y);
          c[q][(k1 + 8 * k2) * pitch[q]] = make_float2(w.x * f, w.y * f);
        }
      }
    __syncwarp();  // the groups' columns, multiplied, back in memory in index order
#pragma unroll
    for (int q = 0; q < 2; q++)
#pragma unroll
      for (int j1 = 0; j1 < 8; j1++)
        v[q][j1] = (L[q].active && j1 < m[q]) ? c[q][(m[q] * l + j1) * pitch[q]]
                                              : make_float2(0.f, 0.f);
    __syncwarp();
    sf8_dft(v[0], m[0], mmax, 1.f, T);
    sf8_dft(v[1], m[1], mmax, 1.f, T);
#pragma unroll
    for (int q = 0; q < 2; q++)
#pragma unroll
      for (int k2 = 0; k2 < 8; k2++)
        if (L[q].active && k2 < m[q]) c[q][(k1 + 8 * k2) * pitch[q]] = v[q][k2];
    if (energy) {
#pragma unroll
      for (int q = 0; q < 2; q++) {
        // the group's eight lane sums in a fixed order
        double t = e[q];
        t += __shfl_xor_sync(0xffffffffu, t, 1);
        t += __shfl_xor_sync(0xffffffffu, t, 2);
        t += __shfl_xor_sync(0xffffffffu, t, 4);
        if (L[q].active && l == 0) a.epart[q == 0 ? u0 : u1] = t;
      }
    }
  }
  cg::this_grid().sync();
  ypass(1.f);
  cg::this_grid().sync();
  // x rows: c2r into the real grid
  SF_FOR_LINE_PAIRS(xrow_first[a.nsys], u0, u1) {
    SfLine L[2] = {sf_line(xrow_first, a.nsys, u0), sf_line(xrow_first, a.nsys, u1)};
    float2 v[2][8];
    int m[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const BatchSys& S = a.sys[L[q].s];
      const int Mx = S.b.M[0], Hx = Mx / 2 + 1;
      m[q] = L[q].active ? Mx / 8 : 1;
      const float2* c = a.rhok + S.kgrid_off + (long long)L[q].r * Hx;
#pragma unroll
      for (int j1 = 0; j1 < 8; j1++) {
        const int j = m[q] * l + j1;
        float2 t = make_float2(0.f, 0.f);
        if (L[q].active && j1 < m[q]) {
          if (j < Hx) {
            t = c[j];
            if (j == 0 || j == Mx / 2) t.y = 0.f;  // FFTW's c2r ignores these imaginary parts
          } else {
            t = c[Mx - j];
            t.y = -t.y;
          }
        }
        v[q][j1] = t;
      }
    }
    const int mmax = sf_warp_mmax(max(m[0], m[1]));
    sf8_dft(v[0], m[0], mmax, 1.f, T);
    sf8_dft(v[1], m[1], mmax, 1.f, T);
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const BatchSys& S = a.sys[L[q].s];
      const int Mx = S.b.M[0];
      float* o = out + S.grid_off + (long long)L[q].r * Mx;
#pragma unroll
      for (int k2 = 0; k2 < 8; k2++)
        if (L[q].active && k2 < m[q]) o[k1 + 8 * k2] = v[q][k2].x;
    }
  }
  if (energy) {  // each system's column energies by one warp: lane-strided sums, then a tree
    const int lane = threadIdx.x & 31;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < a.nsys;
         s += (gridDim.x * blockDim.x) >> 5) {
      double e = 0.0;
      for (int u = a.zcol_first[s] + lane; u < a.zcol_first[s + 1]; u += 32) e += a.epart[u];
      e = warp_sum(e);
      if (lane == 0) a.energy[s] = a.sys[s].efac * e;
    }
  }
}
#undef SF_FOR_LINE_PAIRS

}  // namespace gse
