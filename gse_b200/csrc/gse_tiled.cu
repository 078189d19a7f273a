// gse_tiled.cu -- the tiled spread and gather kernels of the GSE-k path.
//
//  binning   atoms are counting-sorted by (z cell, y cell, x-bin of 4 or 16 cells)
//            of their stencil centre round(x/h) mod M; the FP64 form keeps the
//            original order within a bin so that its sums run in a fixed
//            order, the mixed form's integer sums need no order.
//  spread    CpuGaussCharge::spreadChargeToGrid (CpuGaussCharge.cpp:235-384).
//            FP64 form: output-stationary.  A CTA owns a kTX x kTY x TZ block
//            of the grid; each thread owns one (x, y) column of it with TZ
//            accumulators in registers.  The atoms whose (2n+1)^3 cube reaches
//            the block stream through shared memory in chunks; each warp keeps
//            the ones that touch its 8 x 4 column patch and adds their 2n+1 z
//            weights into its registers.  No atomics; every grid point is
//            written once.  Mixed form: atom-stationary scatter into an int32
//            shared brick tile, added into an int64 grid (scatter_brick).
//  gather    CpuGaussCharge::interpolateLoop (CpuGaussCharge.cpp:105-172): a
//            CTA owns the atoms of a kGX x kGY x kGZ-cell brick and stages the
//            potential of the brick plus its n-cell halo in shared memory;
//            kGatherLanes lanes per atom, over the non-empty (y, z) rows of
//            its sphere.
#include <atomic>
#include <type_traits>

#include <cooperative_groups.h>

#include "gse_internal.cuh"
#include "gse_smallfft.cuh"
#include "gse_tiled.cuh"
#include "gse_tiled_dev.cuh"

namespace gse {

// ===========================================================================
// Binning
// ===========================================================================
template <typename CT>
__global__ void k_bin_count(const typename Vec4<CT>::type* __restrict__ xyzq, int n, BinLayout b,
                            CT inv_hx, CT inv_hy, CT inv_hz, int* __restrict__ key,
                            int* __restrict__ counts, unsigned* __restrict__ qmax_bits,
                            int* __restrict__ bad, long long* __restrict__ clear,
                            long long clear_n, int* __restrict__ rank) {
  pdl_trigger();
  if (clear) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long first = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (long long i = first; i < clear_n / 2; i += stride)
      reinterpret_cast<int4*>(clear)[i] = make_int4(0, 0, 0, 0);
    if ((clear_n & 1) && first == 0) clear[clear_n - 1] = 0;
  }
  float qm = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const auto a = xyzq[i];
    if (bad && !(isfinite(a.x) && isfinite(a.y) && isfinite(a.z) && isfinite(a.w)))
      *bad = kFlagNonFinite;  // the bin below is still in range (wrap1 of any int)
    qm = fmaxf(qm, fabsf((float)a.w));
    const int cx = wrap1(centre_cell(a.x, inv_hx), b.M[0]);
    const int cy = wrap1(centre_cell(a.y, inv_hy), b.M[1]);
    const int cz = wrap1(centre_cell(a.z, inv_hz), b.M[2]);
    const int k = (cz * b.M[1] + cy) * b.nbx + (cx >> b.bxs);
    key[i] = k;
    // rank: the atom's place among its bin's atoms (counting order; the mixed
    // form's consumers are order-free), so the placement needs no atomics
    const int r = atomicAdd(&counts[k], 1);
    if (rank) rank[i] = r;
  }
  if (!qmax_bits) return;  // uniform
  // block maximum first: one atomic per block, not per warp, on the single
  // address (same-address atomics serialise)
  __shared__ float wmax[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) qm = fmaxf(qm, __shfl_xor_sync(0xffffffffu, qm, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = qm;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) qm = fmaxf(qm, wmax[w]);
    // non-negative floats order like their bit patterns (NaN compares largest)
    atomicMax(qmax_bits, __float_as_uint(qm));
  }
}

// Three-phase exclusive scan of counts[0..nb) into start[0..nb].
constexpr int kScanPer = 4;
constexpr int kScanThreads = 1024;
constexpr int kScanTile = kScanPer * kScanThreads;

__global__ void __launch_bounds__(kScanThreads)
    k_scan_tiles(const int* __restrict__ counts, int nb, int* __restrict__ start,
                 int* __restrict__ tile_sums) {
  pdl_trigger();
  pdl_wait();
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanPer;
  int v[kScanPer];
  int s = 0;
#pragma unroll
  for (int j = 0; j < kScanPer; j++) {
    v[j] = (base + j < nb) ? counts[base + j] : 0;
    s += v[j];
  }
  int total;
  int run = block_exclusive_scan(s, &total);
#pragma unroll
  for (int j = 0; j < kScanPer; j++) {
    if (base + j < nb) start[base + j] = run;
    run += v[j];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan_sums(int* __restrict__ tile_sums, int ntiles, int* __restrict__ start, int nb) {
  // ntiles <= kScanTile (checked by the launcher)
  const int base = threadIdx.x * kScanPer;
  int v[kScanPer];
  int s = 0;
#pragma unroll
  for (int j = 0; j < kScanPer; j++) {
    v[j] = (base + j < ntiles) ? tile_sums[base + j] : 0;
    s += v[j];
  }
  int total;
  int run = block_exclusive_scan(s, &total);
#pragma unroll
  for (int j = 0; j < kScanPer; j++) {
    if (base + j < ntiles) tile_sums[base + j] = run;
    run += v[j];
  }
  if (threadIdx.x == 0) start[nb] = total;
}

__global__ void k_scan_add(int* __restrict__ start, int nb, const int* __restrict__ tile_sums) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nb) start[i] += tile_sums[i / kScanTile];
}

// Unordered placement: fill[] counts up from zero per bin.
__global__ void k_bin_place_any(int n, const int* __restrict__ key, const int* __restrict__ start,
                                int* __restrict__ fill, int* __restrict__ tmp) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = key[i];
    tmp[start[k] + atomicAdd(&fill[k], 1)] = i;
  }
}

// Placement in any order within a bin (the mixed form's kernels do not
// depend on the order of the atoms of a bin): counts[] counts down to zero.
template <typename CT>
__global__ void k_bin_place_direct(const typename Vec4<CT>::type* __restrict__ xyzq, int n,
                                   const int* __restrict__ key, const int* __restrict__ start,
                                   int* __restrict__ counts,
                                   typename Vec4<CT>::type* __restrict__ sorted,
                                   int* __restrict__ perm) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = key[i];
    const int slot = start[k] + atomicSub(&counts[k], 1) - 1;
    sorted[slot] = xyzq[i];
    perm[slot] = i;
  }
}

// Order-free placement of the mixed form after a tile-local scan: the block's
// copy of the tile offsets (exclusive prefix of the tile sums) turns the local
// bin starts into global ones; each atom goes to its bin's start plus the rank
// the counting kernel gave it, the global starts are written for the kernels
// that read the bins, and counts[] is cleared for the next call.
__global__ void __launch_bounds__(256)
    k_bin_place_final(const float4* __restrict__ xyzq, int n, const int* __restrict__ key,
                      const int* __restrict__ lstart, const int* __restrict__ tile_sums,
                      int ntiles, int* __restrict__ counts, float4* __restrict__ sorted,
                      int* __restrict__ perm, int* __restrict__ start, int nb,
                      const int* __restrict__ rank) {
  pdl_trigger();
  pdl_wait();
  __shared__ int off[kScanTile];
  constexpr int PER = kScanTile / 256;
  {
    const int base = threadIdx.x * PER;
    int v[PER];
    int s = 0;
#pragma unroll
    for (int j = 0; j < PER; j++) {
      v[j] = base + j < ntiles ? tile_sums[base + j] : 0;
      s += v[j];
    }
    int run = block_exclusive_scan(s, nullptr);
#pragma unroll
    for (int j = 0; j < PER; j++) {
      off[base + j] = run;
      run += v[j];
    }
  }
  __syncthreads();
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  for (int i = gtid; i < n; i += gs) {
    const int k = key[i];
    const int slot = lstart[k] + off[k / kScanTile] + rank[i];
    sorted[slot] = xyzq[i];
    perm[slot] = i;
  }
  for (int i = gtid; i < nb; i += gs) {
    start[i] = lstart[i] + off[i / kScanTile];
    counts[i] = 0;  // zero for the next call's counting
  }
  if (gtid == 0) start[nb] = off[ntiles - 1] + tile_sums[ntiles - 1];
}

// Stable placement: an atom's rank in its bin is the number of bin members
// with a smaller original index.
template <typename CT>
__global__ void k_bin_place_stable(const typename Vec4<CT>::type* __restrict__ xyzq, int n,
                                   const int* __restrict__ key, const int* __restrict__ start,
                                   const int* __restrict__ tmp,
                                   typename Vec4<CT>::type* __restrict__ sorted,
                                   int* __restrict__ perm) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = key[i];
    const int s = start[k], e = start[k + 1];
    int r = 0;
    for (int j = s; j < e; j++) r += (tmp[j] < i);
    sorted[s + r] = xyzq[i];
    perm[s + r] = i;
  }
}

// ===========================================================================
// Spread
// ===========================================================================
// Accumulator / z-weight types of the spread.  FP64 form: double
// accumulators and weights.  Mixed form: the z weights are int32 fixed point
// (kWzBits fraction bits), the (x, y) factor t = q pref wx wy is rounded to
// int32 with a per-launch scale, and each product t_int * wz_int is added
// exactly into an int64 accumulator (one mad.wide.s32), so the grid sum is
// independent of the order of the contributions.
template <typename CT> struct SpreadTypes;
template <> struct SpreadTypes<double> {
  typedef double Acc;
  typedef double Wz;
  typedef double T;
};
template <> struct SpreadTypes<float> {
  typedef long long Acc;
  typedef int Wz;
  typedef int T;
};
constexpr int kWzBits = 26;

__device__ __forceinline__ double madd(double t, double w, double a) { return fma(t, w, a); }
__device__ __forceinline__ long long madd(int t, int w, long long a) {
  return a + (long long)t * (long long)w;
}

template <typename CT>
struct SpreadRec {
  int s[3];                                // first stencil cell relative to the block origin
  CT qp;                                   // q * (2 pi sigma^2)^(-3/2)
  CT w[2][kWPad];                          // x and y weights
  typename SpreadTypes<CT>::Wz wz[kWPad];  // z weights (fixed point in the mixed form)
};

// acc[OZ + k] += t * wz[k] for the k that land inside the block (compile-time
// indices, so the accumulators stay in registers).
template <typename A, typename T, typename WZ, int TZ, int W, int OZ>
__device__ __forceinline__ void add_column(A (&acc)[TZ], T t, const WZ (&wz)[kWPad]) {
#pragma unroll
  for (int k = 0; k < W; k++) {
    if (OZ + k >= 0 && OZ + k < TZ) acc[OZ + k] = madd(t, wz[k], acc[OZ + k]);
  }
}

#define GSE_ZC(i) \
  case i: add_column<A, T, WZ, TZ, W, (i) - (W - 1)>(acc, t, wz); break;
#define GSE_ZC8(i) GSE_ZC(i) GSE_ZC(i + 1) GSE_ZC(i + 2) GSE_ZC(i + 3) GSE_ZC(i + 4) GSE_ZC(i + 5) \
  GSE_ZC(i + 6) GSE_ZC(i + 7)

// The block-relative z offset oz is the same for the whole warp: one
// indirect branch selects the unrolled case.
template <typename A, typename T, typename WZ, int TZ, int W>
__device__ __forceinline__ void add_column_dispatch(int oz, A (&acc)[TZ], T t,
                                                    const WZ (&wz)[kWPad]) {
  static_assert(TZ + W - 1 <= 96, "z dispatch covers 96 offsets");
  switch (oz + W - 1) {
    GSE_ZC8(0) GSE_ZC8(8) GSE_ZC8(16) GSE_ZC8(24) GSE_ZC8(32) GSE_ZC8(40)
    GSE_ZC8(48) GSE_ZC8(56) GSE_ZC8(64) GSE_ZC8(72) GSE_ZC8(80) GSE_ZC8(88)
    default: break;
  }
}
#undef GSE_ZC8
#undef GSE_ZC

// 1-D weights w[j] = exp(-(dc + (j - n) h)^2 / (2 sigma^2)), j < W = 2n+1,
// where dc = c h - x is the offset of the stencil centre (the reference's
// d0 + j h with d0 = (c - n) h - x, CpuGaussCharge.cpp:311-329).  Evaluated
// outward from the centre by the exact ratio recurrence
//   w[n+k] = w[n+k-1] ru[k-1],  ru[k] = ru[k-1] exp(-2 h^2/(2 sigma^2)),
// and the mirror image below the centre.  The decay factor is applied as an
// unevaluated sum hi + lo so that its rounding does not compound.
template <typename CT, int W>
__device__ __forceinline__ void gauss_row(CT dc, CT h, CT inv_2s2, CT dec_hi, CT dec_lo,
                                          CT (&w)[kWPad]) {
  constexpr int n = (W - 1) / 2;
  const CT wc = gexp(mul_rn(mul_rn(-dc, dc), inv_2s2));
  const CT hh = h * h;
  CT ru = gexp(-(2 * dc * h + hh) * inv_2s2);   // w[n+1] / w[n]
  CT rd = gexp(-(hh - 2 * dc * h) * inv_2s2);   // w[n-1] / w[n]
  w[n] = wc;
  CT wu = wc, wd = wc;
#pragma unroll
  for (int k = 1; k <= n; k++) {
    wu *= ru;
    wd *= rd;
    w[n + k] = wu;
    w[n - k] = wd;
    ru = fma(ru, dec_hi, ru * dec_lo);
    rd = fma(rd, dec_hi, rd * dec_lo);
  }
#pragma unroll
  for (int j = W; j < kWPad; j++) w[j] = (CT)0;
}

template <typename CT, int TZ, int W>
__global__ void __launch_bounds__(kSpreadThreads)
    k_spread_tiled(const typename Vec4<CT>::type* __restrict__ sorted,
                   const int* __restrict__ start, const unsigned* __restrict__ qmax_bits,
                   BinLayout b, Stencil<CT> s, Decay<CT> dec, CT* __restrict__ grid) {
  constexpr int n = (W - 1) / 2;
  constexpr int CH = sizeof(CT) == 8 ? kSpreadChunk : 2 * kSpreadChunk;
  constexpr int NT = kSpreadThreads;
  constexpr bool FIXED = sizeof(CT) == 4;
  typedef typename Vec4<CT>::type V;
  typedef typename SpreadTypes<CT>::Acc A;
  typedef typename SpreadTypes<CT>::T T;
  typedef typename SpreadTypes<CT>::Wz WZ;
  __shared__ SpreadRec<CT> rec[CH];
  __shared__ int chunk_atom[CH];
  __shared__ short chunk_shift[CH][3];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY, z0 = blockIdx.z * TZ;
  const int ex = min(kTX, b.M[0] - x0), ey = min(kTY, b.M[1] - y0), ez = min(TZ, b.M[2] - z0);
  // warp patch: 8 (x) x 4 (y); lane -> one column
  const int px0 = (warp & 1) * 8, py0 = (warp >> 1) * 4;
  const int cx = px0 + (lane & 7), cy = py0 + (lane >> 3);

  // mixed form: t is rounded to int32 at 2^st; choose st so that
  // |q pref| 2^st < 2^31 for every atom of the launch
  int st = 0;
  float tscale = 1.f;
  if (FIXED) {
    const float qpm = __uint_as_float(*qmax_bits) * fabsf((float)s.pref);
    st = 30;
    if (!(qpm < 3.0e38f)) {
      st = 0;
    } else {
      while (st > 0 && qpm * exp2f((float)st) >= 2.0e9f) st--;
    }
    tscale = exp2f((float)st);
  }

  A acc[TZ];
#pragma unroll
  for (int z = 0; z < TZ; z++) acc[z] = (A)0;

  // rows (uy, uz) of the relevant region, unwrapped cell coordinates
  const int ry0 = y0 - n, rz0 = z0 - n;
  const int nry = ey + 2 * n, nrz = ez + 2 * n;
  const int nrows = nry * nrz;
  const int ux_lo = x0 - n, ux_hi = x0 + ex + n;  // [lo, hi)

  for (int rbase = 0; rbase < nrows; rbase += NT) {
    // --- this thread's row: wrapped x segments -> atom ranges ---
    const int r = rbase + tid;
    int seg_a[kMaxSeg], seg_e[kMaxSeg], seg_sh[kMaxSeg];
    int nseg = 0, cnt = 0, shy = 0, shz = 0;
    if (r < nrows) {
      const int uy = ry0 + r % nry, uz = rz0 + r / nry;
      const int ccy = pmod(uy, b.M[1]), ccz = pmod(uz, b.M[2]);
      shy = uy - ccy;
      shz = uz - ccz;
      const int rowkey = (ccz * b.M[1] + ccy) * b.nbx;
      int u = ux_lo;
      while (u < ux_hi && nseg < kMaxSeg) {
        const int cu = pmod(u, b.M[0]);
        const int seg_end = min(ux_hi, u + (b.M[0] - cu));  // end of this period
        const int c1 = cu + (seg_end - u);                  // exclusive cell end
        const int a0 = start[rowkey + (cu >> b.bxs)];
        const int a1 = start[rowkey + ((c1 - 1) >> b.bxs) + 1];
        seg_a[nseg] = a0;
        seg_e[nseg] = a1;
        seg_sh[nseg] = u - cu;
        cnt += a1 - a0;
        nseg++;
        u = seg_end;
      }
    }
    int total;
    const int pos0 = block_exclusive_scan(cnt, &total);
    for (int sub = 0; sub < total; sub += CH) {
      // --- copy this thread's atoms with group positions in [sub, sub+CH) ---
      int p = pos0;
      for (int g = 0; g < nseg; g++) {
        for (int j = seg_a[g]; j < seg_e[g]; j++, p++) {
          if (p >= sub && p < sub + CH) {
            chunk_atom[p - sub] = j;
            chunk_shift[p - sub][0] = (short)seg_sh[g];
            chunk_shift[p - sub][1] = (short)shy;
            chunk_shift[p - sub][2] = (short)shz;
          }
        }
      }
      __syncthreads();
      const int cntc = min(CH, total - sub);
      // --- per-atom records ---
      for (int i = tid; i < cntc; i += NT) {
        const V a = sorted[chunk_atom[i]];
        const CT pos[3] = {a.x, a.y, a.z};
        const int org[3] = {x0, y0, z0};
        CT wz[kWPad];
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const int c = centre_cell(pos[d], s.inv_h[d]);
          const CT dc = sub_rn(mul_rn((CT)c, s.h[d]), pos[d]);
          CT w[kWPad];
          gauss_row<CT, W>(dc, s.h[d], s.inv_2s2, dec.hi[d], dec.lo[d], w);
          if (d < 2) {
#pragma unroll
            for (int j = 0; j < kWPad; j++) rec[i].w[d][j] = w[j];
          } else {
#pragma unroll
            for (int j = 0; j < kWPad; j++) wz[j] = w[j];
          }
          rec[i].s[d] = pmod(c, s.M[d]) + chunk_shift[i][d] - n - org[d];
        }
#pragma unroll
        for (int j = 0; j < kWPad; j++) {
          if (FIXED)
            rec[i].wz[j] = (WZ)__float2int_rn((float)wz[j] * (float)(1 << kWzBits));
          else
            rec[i].wz[j] = (WZ)wz[j];
        }
        rec[i].qp = a.w * s.pref;
      }
      __syncthreads();
      // --- each warp: atoms that touch its patch ---
      for (int base = 0; base < cntc; base += 32) {
        const int i = base + lane;
        bool rel = false;
        if (i < cntc) {
          const int sx = rec[i].s[0], sy = rec[i].s[1], sz = rec[i].s[2];
          rel = sx <= px0 + 7 && sx + W - 1 >= px0 && sy <= py0 + 3 && sy + W - 1 >= py0 &&
                sz <= ez - 1 && sz + W - 1 >= 0;
        }
        unsigned mask = __ballot_sync(0xffffffffu, rel);
        while (mask) {
          const int ia = base + __ffs(mask) - 1;
          mask &= mask - 1;
          const int kx = cx - rec[ia].s[0], ky = cy - rec[ia].s[1];
          CT tf = (CT)0;
          if ((unsigned)kx < (unsigned)W && (unsigned)ky < (unsigned)W)
            tf = rec[ia].qp * rec[ia].w[0][kx] * rec[ia].w[1][ky];
          T t;
          if (FIXED)
            t = (T)__float2int_rn((float)tf * tscale);
          else
            t = (T)tf;
          WZ wz[kWPad];
#pragma unroll
          for (int k = 0; k < kWPad; k++) wz[k] = rec[ia].wz[k];
          add_column_dispatch<A, T, WZ, TZ, W>(rec[ia].s[2], acc, t, wz);
        }
      }
      __syncthreads();
    }
  }
  // --- write the block: every point exactly once ---
  if (cx < ex && cy < ey) {
    CT* col = grid + (long long)(x0 + cx) + (long long)(y0 + cy) * b.M[0];
    const long long zs = (long long)b.M[0] * b.M[1];
    const double unscale = FIXED ? exp2(-(double)(st + kWzBits)) : 1.0;
#pragma unroll
    for (int z = 0; z < TZ; z++) {
      if (z < ez) {
        if (FIXED)
          col[(long long)(z0 + z) * zs] = (CT)((double)acc[z] * unscale);
        else
          col[(long long)(z0 + z) * zs] = (CT)acc[z];
      }
    }
  }
}

// ===========================================================================
// Mixed-form spread: atom-stationary scatter into a shared int32 brick tile
// ===========================================================================
// A CTA owns the atoms of one kSB^3-cell brick and a shared tile of the brick
// plus its n-cell halo, T = kSB + 2n points per axis, in int32 fixed point at
// a power-of-two scale 2^S chosen for this brick so that no partial sum can
// overflow (|q| pref summed over the brick's atoms, times 2^S, stays below
// 2^30, and every single contribution below 2^22).  One warp per atom: lanes
// take (x, z) pairs of the (2n+1)^2 plane, form t = q pref wx wz 2^S and add
// round(t wy) for each of the 2n+1 y values -- one fma (rounding by the
// 1.5 * 2^23 magic constant) and one shared-memory integer reduction per cube
// point.  The z-plane pitch is congruent to 2n+1 mod 32, so the 32 lanes of an
// instruction (consecutive (x, z) pairs) hit 32 different banks.
// The finished tile is added into an int64 grid at the common scale
// 2^kFlushBits (S <= kFlushBits, so the shift is exact) by integer
// reductions; integer sums do not depend on their order, so the grid is the
// same bit for bit on every run.
template <int W>
__device__ __forceinline__ void scatter_brick(const float4* __restrict__ sorted,
                                              const int* __restrict__ start, const BinLayout& b,
                                              const Stencil<float>& s, int bxi, int byi, int bzi,
                                              int* __restrict__ tile,
                                              long long* __restrict__ grid64) {
  typedef ScatterGeom<W> G;
  constexpr int n = G::n;
  constexpr int NT = kScatterThreads, NW = NT / 32;
  constexpr int NPASS = (W * W + 31) / 32;
  __shared__ int rng_a[kSB * kSB], rng_p[kSB * kSB];
  __shared__ int alist[kScatterList];
  __shared__ __align__(16) float wys[NW][16];  // each warp's atom's y weights

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int x0 = bxi * kSB, y0 = byi * kSB, z0 = bzi * kSB;
  const float apref = fabsf(s.pref);
  int total;
  const int shift = brick_prologue<W, NT>(
      start, b, x0, y0, z0, tile, rng_a, rng_p,
      [&](int i) { return fabsf(sorted[i].w) * apref; }, &total);
  const float tscale = exp2f((float)shift);

  // per-lane (x, z) pair of each pass and its tile offset: the same for all atoms
  int poff[NPASS], psx[NPASS], psz[NPASS];
#pragma unroll
  for (int pass = 0; pass < NPASS; pass++) {
    const int p = pass * 32 + lane;
    const int pz = p < W * W ? p / W : 0, px = p < W * W ? p - (p / W) * W : 0;
    psx[pass] = px;
    psz[pass] = pz;
    poff[pass] = pz * G::PP + px;
  }

  for (int c0 = 0; c0 < total; c0 += kScatterList) {
    brick_atom_list<NT, kSB * kSB>(rng_a, rng_p, total, c0, kScatterList, alist);
    __syncthreads();
    const int nc = min(kScatterList, total - c0);
    for (int q = warp; q < nc; q += NW) {
      const float4 a = sorted[alist[q]];
      const float pos3[3] = {a.x, a.y, a.z};
      const int org[3] = {x0, y0, z0};
      int loc[3];
      float wl[3];  // lane j < W: weight j along each axis
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const int c = centre_cell(pos3[d], s.inv_h[d]);
        loc[d] = wrap1(c, s.M[d]) - org[d];  // window start in tile coordinates
        const float dd = sub_rn(mul_rn((float)(c - n + lane), s.h[d]), pos3[d]);
        wl[d] = (lane < W) ? wexp(mul_rn(mul_rn(-dd, dd), s.inv_2s2)) : 0.f;
      }
      // every lane needs all W y weights: stored once by the lanes that formed
      // them and read back by four 16-byte broadcast loads (13 shuffles took
      // the shared-memory pipe the reductions wait for; the x and z weights,
      // one each per pass, stay shuffles: per-lane loads of them were slower)
      float wy[W];
      {
        __syncwarp();  // the warp's previous atom has read its weights
        if (lane < 16) wys[warp][lane] = wl[1];
        __syncwarp();
        const float4* v = reinterpret_cast<const float4*>(wys[warp]);
#pragma unroll
        for (int q4 = 0; q4 < (W + 3) / 4; q4++) {
          const float4 t = v[q4];
          wy[4 * q4] = t.x;
          if (4 * q4 + 1 < W) wy[4 * q4 + 1] = t.y;
          if (4 * q4 + 2 < W) wy[4 * q4 + 2] = t.z;
          if (4 * q4 + 3 < W) wy[4 * q4 + 3] = t.w;
        }
      }
      // y weights in pairs for the packed fma (two points per instruction)
      unsigned long long wy2[W / 2];
#pragma unroll
      for (int k = 0; k + 1 < W; k += 2)
        asm("mov.b64 %0, {%1, %2};" : "=l"(wy2[k / 2]) : "f"(wy[k]), "f"(wy[k + 1]));
      unsigned long long magic2;
      asm("mov.b64 %0, {%1, %1};" : "=l"(magic2) : "f"(12582912.0f));
      const float qp = a.w * s.pref * tscale;
      int* base = tile + loc[2] * G::PP + loc[1] * G::RP + loc[0];
#pragma unroll
      for (int pass = 0; pass < NPASS; pass++) {
        const float wx = __shfl_sync(0xffffffffu, wl[0], psx[pass]);
        const float wz = __shfl_sync(0xffffffffu, wl[2], psz[pass]);
        if (pass * 32 + lane < W * W) {
          const float t = qp * wx * wz;
          int* cell = base + poff[pass];
          unsigned long long t2;
          asm("mov.b64 %0, {%1, %1};" : "=l"(t2) : "f"(t));
#pragma unroll
          for (int k = 0; k + 1 < W; k += 2) {
            // round(t wy) for two points: |t wy| < 2^22, so 1.5*2^23 + t wy has
            // unit spacing (each half rounded once, as fmaf does)
            unsigned long long r2;
            asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r2) : "l"(t2), "l"(wy2[k / 2]), "l"(magic2));
            unsigned lo, hi;
            asm("mov.b64 {%0, %1}, %2;" : "=r"(lo), "=r"(hi) : "l"(r2));
            atomicAdd(cell + k * G::RP, (int)lo - 0x4B400000);
            atomicAdd(cell + (k + 1) * G::RP, (int)hi - 0x4B400000);
          }
          {
            const int v = __float_as_int(fmaf(t, wy[W - 1], 12582912.0f)) - 0x4B400000;
            atomicAdd(cell + (W - 1) * G::RP, v);
          }
        }
      }
    }
    __syncthreads();
  }
  brick_flush<W, NT>(tile, b, x0, y0, z0, shift, grid64);
}

template <int W>
__global__ void __launch_bounds__(kScatterThreads)
    k_spread_scatter(const float4* __restrict__ sorted, const int* __restrict__ start,
                     BinLayout b, Stencil<float> s, long long* __restrict__ grid64) {
  pdl_trigger();
  pdl_wait();
  extern __shared__ int tile[];
  scatter_brick<W>(sorted, start, b, s, blockIdx.x, blockIdx.y, blockIdx.z, tile, grid64);
}

// float grid from the int64 accumulation grid at 2^kFlushBits
__global__ void k_grid64_to_real(const long long* __restrict__ g64, long long size,
                                 float* __restrict__ out) {
  const double unscale = exp2(-(double)kFlushBits);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < size;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)((double)g64[i] * unscale);
}

// ===========================================================================
// Gather
// ===========================================================================
// Sphere test of one stencil point.  FP64 form: the reference's own sum and
// order, (dx^2 + dy^2) + dz^2 < rcut^2 (CpuGaussCharge.cpp:157-158), so the
// point set is bit-identical.  Mixed form: dx^2 < rcut^2 - (dy^2 + dz^2).
template <typename CT>
__device__ __forceinline__ bool in_sphere(CT dx2, CT dy2, CT dz2, CT rem, CT rcut2);
template <>
__device__ __forceinline__ bool in_sphere<double>(double dx2, double dy2, double dz2, double,
                                                  double rcut2) {
  return add_rn(add_rn(dx2, dy2), dz2) < rcut2;
}
template <>
__device__ __forceinline__ bool in_sphere<float>(float dx2, float, float, float rem, float) {
  return dx2 < rem;
}

// s0 = sum_k m_k wx[k] row[k], s1 = sum_k m_k wx[k] dx[k] row[k] over the
// 2n+1 points of one stencil row, m_k the sphere test.  The test guards the
// two fmas (predicated, no select); a skipped point adds exactly nothing.
template <typename CT, int W, int K0 = 0, int K1 = W>
__device__ __forceinline__ void row_sums(const CT* row, const CT (&dx2)[W], const CT (&wx)[W],
                                         const CT (&wdx)[W], CT dy2, CT dz2, CT rem, CT rcut2,
                                         CT& s0, CT& s1) {
  CT a = (CT)0, c = (CT)0;
#pragma unroll
  for (int k = K0; k < K1; k++) {
    const CT ph = row[k];
    if (in_sphere<CT>(dx2[k], dy2, dz2, rem, rcut2)) {
      a = fma(wx[k], ph, a);
      c = fma(wdx[k], ph, c);
    }
  }
  s0 = a;
  s1 = c;
}

// Shared memory of the gather for calculation type CT and stencil width W:
// the potential tile [TZ][ZP] (rows of pitch TP), per-atom weight tables and
// per-atom row lists.
template <typename CT, int W, int NT = kGatherThreads, int GL = kGatherLanes>
struct GatherGeom {
  static constexpr int n = (W - 1) / 2;
  static constexpr int TX = kGX + 2 * n, TY = kGY + 2 * n, TZ = kGZ + 2 * n;
  static constexpr int TP = TX | 1;  // odd row pitch
  // plane pitch = W*TP (mod 32): row (jy, jz) starts in bank TP*(jy + W*jz)
  // mod 32, distinct for 32 consecutive (jy, jz)
  static constexpr int ZP = ((TY * TP + 31) / 32) * 32 + ((W * TP) % 32);
  static constexpr int NW = NT / 32;
  static constexpr int APW = 32 / GL;  // atoms per warp at a time
  static constexpr size_t bytes =
      sizeof(CT) * (TZ * ZP + NW * APW * 9 * kWPad) + sizeof(int) * NW * APW * W * W;
};

// The gather of the atoms of one brick by a block of NT threads.  kGatherLanes
// lanes share one atom (two atoms per warp at 16): each group builds its
// atom's weight tables, compacts the (y, z) rows that meet the sphere and sums
// them, one row per lane and iteration, in the order of the row list.  GL
// lanes per atom (16 by default; the batched launch may take 8).
template <typename CT, int W, int NT = kGatherThreads, int GL = kGatherLanes>
__device__ __forceinline__ void gather_brick(const typename Vec4<CT>::type* __restrict__ sorted,
                                             const int* __restrict__ perm,
                                             const int* __restrict__ start, const BinLayout& b,
                                             const Stencil<CT>& s, const CT* __restrict__ phi,
                                             double outscale, double* __restrict__ fx,
                                             double* __restrict__ fy, double* __restrict__ fz,
                                             int bxi, int byi, int bzi, unsigned char* gsm) {
  typedef GatherGeom<CT, W, NT, GL> GG;
  constexpr int n = GG::n, TX = GG::TX, TY = GG::TY, TZ = GG::TZ, TP = GG::TP, ZP = GG::ZP;
  constexpr int NW = GG::NW, APW = GG::APW;
  constexpr int NR = kGY * kGZ;  // cell rows of the brick
  constexpr int NG = (W * W + GL - 1) / GL;
  static_assert(TZ * ZP < (1 << 23), "tile offsets fit the row list entries");
  typedef typename Vec4<CT>::type V;
  CT* tile = (CT*)gsm;                                   // [TZ][ZP]
  CT* tabs = tile + TZ * ZP;                             // [NW][APW][axis][d, d^2, w][kWPad]
  int* rowl = (int*)(tabs + NW * APW * 9 * kWPad);       // [NW][APW][W*W]
  __shared__ int rng_a[NR], rng_p[NR + 1];
  __shared__ int alist[kGatherList];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grp = lane / GL, gl = lane % GL;
  const int x0 = bxi * kGX, y0 = byi * kGY, z0 = bzi * kGZ;
  const int ex = min(kGX, b.M[0] - x0), ey = min(kGY, b.M[1] - y0), ez = min(kGZ, b.M[2] - z0);

  // atoms of the brick: one range per (y, z) cell row
  int cnt = 0;
  if (tid < NR) {
    const int yy = tid % kGY, zz = tid / kGY;
    int a0 = 0, a1 = 0;
    if (yy < ey && zz < ez) {
      const int rowkey = ((z0 + zz) * b.M[1] + (y0 + yy)) * b.nbx;
      a0 = start[rowkey + (x0 >> b.bxs)];
      a1 = start[rowkey + ((x0 + ex - 1) >> b.bxs) + 1];
    }
    rng_a[tid] = a0;
    cnt = a1 - a0;
  }
  int natoms;
  const int pos = block_exclusive_scan(cnt, &natoms);
  if (tid < NR) rng_p[tid] = pos;
  if (tid == 0) rng_p[NR] = natoms;
  if (natoms == 0) return;  // uniform: natoms is the same in every thread

  // potential of the brick plus halo, staged by asynchronous element copies
  // so that a warp keeps all of its rows in flight
  stage_tile_async<CT, TX, TY, TZ, TP, ZP, NW>(phi, b, x0, y0, z0, n, tile);
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();

  CT* tb = tabs + (warp * APW + grp) * 9 * kWPad;  // [axis][d, d^2, w][j]
  int* rl = rowl + (warp * APW + grp) * W * W;
  // (jy, jz) of the rows each lane tests, the same for every atom: first the
  // (W-1)^2 rows with jy, jz >= 1, then the 2W-1 rows with jy = 0 or jz = 0,
  // which lie outside the sphere whenever dy^2 (dz^2) at index 0 is at least
  // rcut^2 -- for every atom when n h exceeds rcut by more than rounding
  constexpr int NI = (W - 1) * (W - 1);
  constexpr int NGI = (NI + GL - 1) / GL;  // groups that hold the inner rows
  // (jy, jz) of candidate row r (formed where it is used: a table of them
  // would hold 2 NG registers through the whole atom loop)
  auto cand = [&](int r, int& jy, int& jz) {
    if (r < NI) {
      jz = 1 + r / (W - 1);
      jy = 1 + r % (W - 1);
    } else if (r < NI + W) {
      jz = r - NI;
      jy = 0;
    } else if (r < W * W) {
      jz = 0;
      jy = r - NI - W + 1;
    } else {
      jz = jy = 0;
    }
  };
  const unsigned gmask = GL == 32 ? 0xffffffffu : ((1u << GL) - 1u);
  for (int c0 = 0; c0 < natoms; c0 += kGatherList) {
    brick_atom_list<NT, NR>(rng_a, rng_p, natoms, c0, kGatherList, alist);
    __syncthreads();
    const int nc = min(kGatherList, natoms - c0);
    // the next atom's record and output slot are loaded one iteration ahead,
    // so their global-memory latency overlaps the current atom's work
    int ai_n = 0, o_n = 0;
    V a_n;
    auto fetch = [&](int qq0) {
      const int qq = qq0 + grp;
      ai_n = alist[qq < nc ? qq : qq0];
      a_n = sorted[ai_n];
      o_n = perm[ai_n];
    };
    if (APW * warp < nc) fetch(APW * warp);
    for (int q0 = APW * warp; q0 < nc; q0 += APW * NW) {
      const int q = q0 + grp;
      const bool valid = q < nc;  // the last group of a chunk may have no atom
      const V a = a_n;
      const int out_slot = o_n;
      if (q0 + APW * NW < nc) fetch(q0 + APW * NW);
      const CT pos3[3] = {a.x, a.y, a.z};
      const int org[3] = {x0, y0, z0};
      int loc[3];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const int c = centre_cell(pos3[d], s.inv_h[d]);
        loc[d] = wrap1(c, s.M[d]) - org[d];  // first stencil cell in tile coordinates
        for (int j = gl; j < W; j += GL) {
          const CT dd = sub_rn(pos3[d], mul_rn((CT)(c - n + j), s.h[d]));
          const CT d2 = mul_rn(dd, dd);
          tb[(d * 3 + 0) * kWPad + j] = dd;
          tb[(d * 3 + 1) * kWPad + j] = d2;
          tb[(d * 3 + 2) * kWPad + j] = wexp(mul_rn(-d2, s.inv_2s2));
        }
      }
      __syncwarp();
      // the rows with jy = 0 or jz = 0 are tested only when one of the warp's
      // atoms could have one inside (adding dz^2 >= 0 cannot take a sum below
      // dy^2, so dy^2 >= rcut^2 at jy = 0 rules out its whole plane)
      const bool edges = !__all_sync(0xffffffffu, tb[(1 * 3 + 1) * kWPad + 0] >= s.rcut2 &&
                                                      tb[(2 * 3 + 1) * kWPad + 0] >= s.rcut2);
      // non-empty rows (the whole row is outside the sphere when dy^2+dz^2 >= rcut^2)
      int nrow = 0;
#pragma unroll
      for (int g = 0; g < NG; g++) {
        if (g >= NGI && !edges) break;  // warp-uniform
        const int r = g * GL + gl;
        int jy, jz;
        cand(r, jy, jz);
        bool ne = false;
        if (r < W * W)
          ne = add_rn(tb[(1 * 3 + 1) * kWPad + jy], tb[(2 * 3 + 1) * kWPad + jz]) < s.rcut2;
        const unsigned m = (__ballot_sync(0xffffffffu, ne) >> (GL * grp)) & gmask;
        // the row's tile offset with its (jz, jy): bits 8+ offset, 4-7 jz, 0-3 jy
        if (ne) rl[nrow + __popc(m & ((1u << gl) - 1u))] = ((jz * ZP + jy * TP) << 8) | (jz << 4) | jy;
        nrow += __popc(m);
      }
      __syncwarp();
      CT dx2[W], wx[W], wdx[W];
#pragma unroll
      for (int k = 0; k < W; k++) {
        dx2[k] = tb[(0 * 3 + 1) * kWPad + k];
        wx[k] = tb[(0 * 3 + 2) * kWPad + k];
        wdx[k] = wx[k] * tb[(0 * 3 + 0) * kWPad + k];
      }
      // each row's 2n+1 terms and a lane's rows (about rows/16 of them) in CT, the
      // lanes' sums in double (the reference's AT)
      CT lx = 0, ly = 0, lz = 0;
      const CT* abase = tile + loc[2] * ZP + loc[1] * TP + loc[0];  // the atom's first row
      // an end point of the rows lies outside the sphere for every row when
      // dx^2 >= rcut^2 there (rem <= rcut^2): the rows are then summed
      // without it, the same terms in the same order.  The first point is
      // outside for nearly every atom (n h >= rcut), the last for about half.
      const bool head = __any_sync(0xffffffffu, dx2[0] < s.rcut2);
      const bool tail = __any_sync(0xffffffffu, dx2[W - 1] < s.rcut2);
      auto rows = [&](auto k0, auto k1) {
        constexpr int K0 = decltype(k0)::value;
        constexpr int K1 = decltype(k1)::value;
        for (int i = gl; i < nrow; i += GL) {
          const int r = rl[i];
          const int jz = (r >> 4) & 15, jy = r & 15;
          const CT dy2 = tb[(1 * 3 + 1) * kWPad + jy], dz2 = tb[(2 * 3 + 1) * kWPad + jz];
          const CT rem = s.rcut2 - (dy2 + dz2);
          const CT* row = abase + (r >> 8);
          CT s0, s1;
          row_sums<CT, W, K0, K1>(row, dx2, wx, wdx, dy2, dz2, rem, s.rcut2, s0, s1);
          const CT wyz = tb[(1 * 3 + 2) * kWPad + jy] * tb[(2 * 3 + 2) * kWPad + jz];
          lx += wyz * s1;
          ly += wyz * tb[(1 * 3 + 0) * kWPad + jy] * s0;
          lz += wyz * tb[(2 * 3 + 0) * kWPad + jz] * s0;
        }
      };
      if (head)
        rows(std::integral_constant<int, 0>(), std::integral_constant<int, W>());
      else if (tail)
        rows(std::integral_constant<int, 1>(), std::integral_constant<int, W>());
      else
        rows(std::integral_constant<int, 1>(), std::integral_constant<int, W - 1>());
      double ax = (double)lx, ay = (double)ly, az = (double)lz;
#pragma unroll
      for (int o = GL / 2; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
      }
      if (gl == 0 && valid) {
        const double f = outscale * (double)(a.w * s.pref);
        fx[out_slot] = f * ax;
        fy[out_slot] = f * ay;
        fz[out_slot] = f * az;
      }
      __syncwarp();
    }
    __syncthreads();
  }
}

template <typename CT, int W>
__global__ void __launch_bounds__(kGatherThreads, sizeof(CT) == 4 ? 2 : 1)
    k_gather_tiled(const typename Vec4<CT>::type* __restrict__ sorted,
                   const int* __restrict__ perm, const int* __restrict__ start, BinLayout b,
                   Stencil<CT> s, const CT* __restrict__ phi, double outscale,
                   double* __restrict__ fx, double* __restrict__ fy, double* __restrict__ fz) {
  pdl_wait();
  extern __shared__ __align__(16) unsigned char gsm[];
  gather_brick<CT, W>(sorted, perm, start, b, s, phi, outscale, fx, fy, fz, blockIdx.x,
                      blockIdx.y, blockIdx.z, gsm);
}

// ===========================================================================
// Launchers
// ===========================================================================
template <typename CT>
cudaError_t launch_bin_sorted(const typename Vec4<CT>::type* xyzq, int n, const BinLayout& b,
                              CT inv_hx, CT inv_hy, CT inv_hz, BinScratch w,
                              typename Vec4<CT>::type* sorted, int* perm, cudaStream_t st) {
  const int nb = b.M[1] * b.M[2] * b.nbx;
  const int ntiles = (nb + kScanTile - 1) / kScanTile;
  if (ntiles > kScanTile) return cudaErrorInvalidValue;
  cudaError_t e = cudaSuccess;
  if (!(sizeof(CT) == 4 && w.counts_zero)) {
    e = cudaMemsetAsync(w.counts, 0, sizeof(int) * nb, st);
    if (e != cudaSuccess) return e;
  }
  // the largest |q| feeds the FP64 spread's range check only
  unsigned* qmax = sizeof(CT) == 8 ? w.qmax_bits : nullptr;
  if (qmax) {
    e = cudaMemsetAsync(qmax, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
  }
  // a grid to clear takes every SM; the atoms alone, one thread each up to that
  const int gb = w.clear ? sm_count() * 8
                         : (int)std::min<long long>(sm_count() * 8,
                                                    (n + 255) / 256 > 0 ? (n + 255) / 256 : 1);
  if (n > 0)
    k_bin_count<CT><<<gb, 256, 0, st>>>(xyzq, n, b, inv_hx, inv_hy, inv_hz, w.key, w.counts,
                                        qmax, w.bad, w.clear, w.clear_n,
                                        (sizeof(CT) == 4 && w.lstart) ? w.tmp : nullptr);
  else if (w.clear)
    e = cudaMemsetAsync(w.clear, 0, sizeof(long long) * w.clear_n, st);
  if (e != cudaSuccess) return e;
  return launch_bin_scan_place<CT>(xyzq, n, nb, w, sorted, perm, st);
}

// counts (filled) -> start offsets -> placement of the atoms: stable (in
// the original order within a bin) for the FP64 form, whose output-stationary
// spread sums atoms in bin order; any order for the mixed form.
template <typename CT>
cudaError_t launch_bin_scan_place(const typename Vec4<CT>::type* xyzq, int n, int nb,
                                  BinScratch w, typename Vec4<CT>::type* sorted, int* perm,
                                  cudaStream_t st) {
  const int ntiles = (nb + kScanTile - 1) / kScanTile;
  if (ntiles > kScanTile) return cudaErrorInvalidValue;
  cudaError_t e;
  const int gb = (int)std::min<long long>(sm_count() * 8, (n + 255) / 256 > 0 ? (n + 255) / 256 : 1);
  if (sizeof(CT) == 4 && w.lstart) {
    // two kernels: tile-local scan, then placement with the tile offsets
    // each kernel follows the previous one of the binning on the stream
    // (the counts, when there are atoms)
    e = launch_dependent(n > 0, k_scan_tiles, dim3(ntiles), dim3(kScanThreads), 0, st, w.counts,
                         nb, w.lstart, w.tile_sums);
    if (e != cudaSuccess) return e;
    e = launch_dependent(true, k_bin_place_final, dim3(gb), dim3(256), 0, st,
                         (const float4*)xyzq, n, (const int*)w.key, (const int*)w.lstart,
                         (const int*)w.tile_sums, ntiles, w.counts, (float4*)sorted, perm,
                         w.start, nb, (const int*)w.tmp);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
  }
  k_scan_tiles<<<ntiles, kScanThreads, 0, st>>>(w.counts, nb, w.start, w.tile_sums);
  k_scan_sums<<<1, kScanThreads, 0, st>>>(w.tile_sums, ntiles, w.start, nb);
  k_scan_add<<<(nb + 255) / 256, 256, 0, st>>>(w.start, nb, w.tile_sums);
  if (n > 0) {
    if (sizeof(CT) == 4) {
      k_bin_place_direct<CT><<<gb, 256, 0, st>>>(xyzq, n, w.key, w.start, w.counts, sorted, perm);
    } else {
      e = cudaMemsetAsync(w.counts, 0, sizeof(int) * nb, st);
      if (e != cudaSuccess) return e;
      k_bin_place_any<<<gb, 256, 0, st>>>(n, w.key, w.start, w.counts, w.tmp);
      k_bin_place_stable<CT><<<gb, 256, 0, st>>>(xyzq, n, w.key, w.start, w.tmp, sorted, perm);
    }
  }
  return cudaGetLastError();
}

template <typename CT, int TZ, int W>
static cudaError_t spread_w(const typename Vec4<CT>::type* sorted, const int* start,
                            const unsigned* qmax_bits, const BinLayout& b, const Stencil<CT>& s,
                            CT* grid, cudaStream_t st) {
  const Decay<CT> dec = make_decay<CT>(s);
  dim3 grd((b.M[0] + kTX - 1) / kTX, (b.M[1] + kTY - 1) / kTY, (b.M[2] + TZ - 1) / TZ);
  k_spread_tiled<CT, TZ, W><<<grd, kSpreadThreads, 0, st>>>(sorted, start, qmax_bits, b, s, dec,
                                                             grid);
  return cudaGetLastError();
}

template <typename CT>
bool spread_tiled_supported(const Stencil<CT>& s) {
  for (int d = 0; d < 3; d++)
    if (s.nst[d] != s.nst[0]) return false;
  const int W = 2 * s.nst[0] + 1;
  return W == 9 || W == 11 || W == 13 || W == 15;
}

template <typename CT>
cudaError_t launch_spread_tiled(const typename Vec4<CT>::type* sorted, const int* start,
                                const unsigned* qmax_bits, const BinLayout& b,
                                const Stencil<CT>& s, CT* grid, cudaStream_t st) {
  constexpr int TZ = sizeof(CT) == 8 ? kTZ64 : kTZ32;
  switch (2 * s.nst[0] + 1) {
    case 9: return spread_w<CT, TZ, 9>(sorted, start, qmax_bits, b, s, grid, st);
    case 11: return spread_w<CT, TZ, 11>(sorted, start, qmax_bits, b, s, grid, st);
    case 13: return spread_w<CT, TZ, 13>(sorted, start, qmax_bits, b, s, grid, st);
    case 15: return spread_w<CT, TZ, 15>(sorted, start, qmax_bits, b, s, grid, st);
  }
  return cudaErrorInvalidValue;
}

template <typename CT, int W>
static cudaError_t gather_w(const typename Vec4<CT>::type* sorted, const int* perm,
                            const int* start, const BinLayout& b, const Stencil<CT>& s,
                            const CT* phi, double outscale, double* fx, double* fy, double* fz,
                            bool pdl, cudaStream_t st) {
  const size_t smem = GatherGeom<CT, W>::bytes;
  static std::atomic<bool> attr[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr[dev]) {
    const cudaError_t e = cudaFuncSetAttribute(
        k_gather_tiled<CT, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr[dev] = true;
  }
  dim3 grd((b.M[0] + kGX - 1) / kGX, (b.M[1] + kGY - 1) / kGY, (b.M[2] + kGZ - 1) / kGZ);
  const cudaError_t e = launch_dependent(pdl, k_gather_tiled<CT, W>, grd, dim3(kGatherThreads),
                                         smem, st, sorted, perm, start, b, s, phi, outscale, fx,
                                         fy, fz);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_gather_tiled(const typename Vec4<CT>::type* sorted, const int* perm,
                                const int* start, const BinLayout& b, const Stencil<CT>& s,
                                const CT* phi, double outscale, double* fx, double* fy,
                                double* fz, bool pdl, cudaStream_t st) {
  switch (2 * s.nst[0] + 1) {
    case 9: return gather_w<CT, 9>(sorted, perm, start, b, s, phi, outscale, fx, fy, fz, pdl, st);
    case 11:
      return gather_w<CT, 11>(sorted, perm, start, b, s, phi, outscale, fx, fy, fz, pdl, st);
    case 13:
      return gather_w<CT, 13>(sorted, perm, start, b, s, phi, outscale, fx, fy, fz, pdl, st);
    case 15:
      return gather_w<CT, 15>(sorted, perm, start, b, s, phi, outscale, fx, fy, fz, pdl, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_grid64_to_real(const long long* grid64, long long size, float* out,
                                  cudaStream_t st) {
  k_grid64_to_real<<<sm_count() * 8, 256, 0, st>>>(grid64, size, out);
  return cudaGetLastError();
}

template <int W>
static cudaError_t scatter_w(const float4* sorted, const int* start, const BinLayout& b,
                             const Stencil<float>& s, long long* grid64, float* rho, bool zeroed,
                             cudaStream_t st) {
  typedef ScatterGeom<W> G;
  const size_t smem = sizeof(int) * G::words;
  static std::atomic<bool> attr[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr[dev]) {
    const cudaError_t e = cudaFuncSetAttribute(
        k_spread_scatter<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr[dev] = true;
  }
  const long long size = (long long)b.M[0] * b.M[1] * b.M[2];
  cudaError_t e = cudaSuccess;
  if (!zeroed) e = cudaMemsetAsync(grid64, 0, sizeof(long long) * size, st);
  if (e != cudaSuccess) return e;
  const int nb[3] = {(b.M[0] + kSB - 1) / kSB, (b.M[1] + kSB - 1) / kSB,
                     (b.M[2] + kSB - 1) / kSB};
  // with the grid cleared earlier the spread follows the binning's last kernel
  e = launch_dependent(zeroed, k_spread_scatter<W>, dim3(nb[0], nb[1], nb[2]),
                       dim3(kScatterThreads), smem, st, sorted, start, b, s, grid64);
  if (e != cudaSuccess) return e;
  // rho == nullptr: the caller converts the int64 grid itself (the own FFT)
  if (rho) k_grid64_to_real<<<sm_count() * 8, 256, 0, st>>>(grid64, size, rho);
  return cudaGetLastError();
}

cudaError_t launch_spread_scatter(const float4* sorted, const int* start, const BinLayout& b,
                                  const Stencil<float>& s, long long* grid64, float* rho,
                                  bool zeroed, cudaStream_t st) {
  switch (2 * s.nst[0] + 1) {
    case 9: return scatter_w<9>(sorted, start, b, s, grid64, rho, zeroed, st);
    case 11: return scatter_w<11>(sorted, start, b, s, grid64, rho, zeroed, st);
    case 13: return scatter_w<13>(sorted, start, b, s, grid64, rho, zeroed, st);
    case 15: return scatter_w<15>(sorted, start, b, s, grid64, rho, zeroed, st);
  }
  return cudaErrorInvalidValue;
}

// ===========================================================================
// Batched systems: persistent kernels over (system, brick) work items
// ===========================================================================
__global__ void k_batch_bin_count(const float4* __restrict__ xyzq, int ntot,
                                  const BatchSys* __restrict__ sys, const int* __restrict__ first,
                                  int nsys, int* __restrict__ key, int* __restrict__ counts) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
    const float4 a = xyzq[i];
    const BatchSys& S = sys[batch_sys_of(first, nsys, i)];
    const int cx = wrap1(centre_cell(a.x, S.sp.inv_h[0]), S.b.M[0]);
    const int cy = wrap1(centre_cell(a.y, S.sp.inv_h[1]), S.b.M[1]);
    const int cz = wrap1(centre_cell(a.z, S.sp.inv_h[2]), S.b.M[2]);
    const int k = S.bin_off + (cz * S.b.M[1] + cy) * S.b.nbx + (cx >> S.b.bxs);
    key[i] = k;
    atomicAdd(&counts[k], 1);
  }
}

template <int W>
__global__ void __launch_bounds__(kScatterThreads)
    k_batch_scatter(const float4* __restrict__ sorted, const int* __restrict__ start,
                    const BatchSys* __restrict__ sys, const BatchItem* __restrict__ items,
                    int nitems, long long* __restrict__ grid64) {
  extern __shared__ int tile[];
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BatchItem item = items[it];
    const BatchSys& S = sys[item.sys];
    scatter_brick<W>(sorted, start + S.bin_off, S.b, S.sp, item.bx, item.by, item.bz, tile,
                     grid64 + S.grid_off);
    __syncthreads();
  }
}

// rhok *= G per bin; energy[s] += efac_s * sum_k G |rho(k)|^2 (full spectrum).
// kfirst: ascending first bins of the systems' spectra, ksys: the system of
// each of those slots (grids are grouped by size, not in system order).
__global__ void __launch_bounds__(256)
    k_batch_green_apply(float2* __restrict__ rhok, const float* __restrict__ tab,
                        long long ktot, const BatchSys* __restrict__ sys,
                        const long long* __restrict__ kfirst, const int* __restrict__ ksys,
                        int nsys, double* __restrict__ energy) {
  const int lane = threadIdx.x & 31;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < ktot;
       base += (long long)gridDim.x * blockDim.x) {
    const long long idx = base + threadIdx.x;
    int s = 0;
    double e = 0.0;
    if (idx < ktot) {
      int lo = 0, hi = nsys - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (kfirst[mid] <= idx) lo = mid; else hi = mid - 1;
      }
      s = ksys[lo];
      const BatchSys& S = sys[s];
      float2 v = rhok[idx];
      const float f = tab[idx];
      const int sx = S.b.M[0] / 2 + 1;
      const int ix = (int)((idx - kfirst[lo]) % sx);
      const double wgt = (ix == 0 || ((S.b.M[0] & 1) == 0 && ix == S.b.M[0] / 2)) ? 1.0 : 2.0;
      const double re = v.x, im = v.y;
      if (energy) e = S.efac * wgt * (double)f * (re * re + im * im);
      v.x *= f;
      v.y *= f;
      rhok[idx] = v;
    }
    if (energy) {
      const int s0 = __shfl_sync(0xffffffffu, s, 0);
      if (__all_sync(0xffffffffu, s == s0)) {
        e = warp_sum(e);
        if (lane == 0 && idx < ktot) atomicAdd(&energy[s0], e);
        else if (lane == 0) atomicAdd(&energy[s0], e);
      } else if (idx < ktot) {
        atomicAdd(&energy[s], e);
      }
    }
  }
}

template <int W>
__global__ void __launch_bounds__(kGatherThreads, 2)
    k_batch_gather(const float4* __restrict__ sorted, const int* __restrict__ perm,
                   const int* __restrict__ start, const BatchSys* __restrict__ sys,
                   const BatchItem* __restrict__ items, int nitems, const float* __restrict__ phi,
                   double outscale, double* __restrict__ fx, double* __restrict__ fy,
                   double* __restrict__ fz) {
  extern __shared__ __align__(16) unsigned char gsm[];
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BatchItem item = items[it];
    const BatchSys& S = sys[item.sys];
    gather_brick<float, W>(sorted, perm, start + S.bin_off, S.b, S.sg, phi + S.grid_off, outscale,
                           fx, fy, fz, item.bx, item.by, item.bz, gsm);
    __syncthreads();
  }
}

template <class K>
static cudaError_t set_max_smem(K kernel, size_t bytes, std::atomic<bool>* done) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (done[dev]) return cudaSuccess;
  const cudaError_t e =
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) done[dev] = true;
  return e;
}

template <int W>
static cudaError_t batch_scatter_w(const float4* sorted, const int* start, const BatchSys* sys,
                                   const BatchItem* items, int nitems, int ctas,
                                   long long* grid64, cudaStream_t st) {
  static std::atomic<bool> done[64];
  const size_t smem = sizeof(int) * ScatterGeom<W>::words;
  const cudaError_t e = set_max_smem(k_batch_scatter<W>, smem, done);
  if (e != cudaSuccess) return e;
  k_batch_scatter<W><<<std::min(ctas, nitems), kScatterThreads, smem, st>>>(sorted, start, sys,
                                                                           items, nitems, grid64);
  return cudaGetLastError();
}

template <int W>
static cudaError_t batch_gather_w(const float4* sorted, const int* perm, const int* start,
                                  const BatchSys* sys, const BatchItem* items, int nitems,
                                  int ctas, const float* phi, double outscale, double* fx,
                                  double* fy, double* fz, cudaStream_t st) {
  static std::atomic<bool> done[64];
  const size_t smem = GatherGeom<float, W>::bytes;
  const cudaError_t e = set_max_smem(k_batch_gather<W>, smem, done);
  if (e != cudaSuccess) return e;
  k_batch_gather<W><<<std::min(ctas, nitems), kGatherThreads, smem, st>>>(
      sorted, perm, start, sys, items, nitems, phi, outscale, fx, fy, fz);
  return cudaGetLastError();
}

cudaError_t launch_batch_bin(const float4* xyzq, int ntot, const BatchSys* sys, const int* first,
                             int nsys, int nbins, BinScratch w, float4* sorted, int* perm,
                             cudaStream_t st) {
  const cudaError_t e = cudaMemsetAsync(w.counts, 0, sizeof(int) * nbins, st);
  if (e != cudaSuccess) return e;
  const int gb = (int)std::min<long long>(sm_count() * 8, (ntot + 255) / 256 > 0 ? (ntot + 255) / 256 : 1);
  if (ntot > 0)
    k_batch_bin_count<<<gb, 256, 0, st>>>(xyzq, ntot, sys, first, nsys, w.key, w.counts);
  return launch_bin_scan_place<float>(xyzq, ntot, nbins, w, sorted, perm, st);
}

cudaError_t launch_batch_spread(const float4* sorted, const int* start, const BatchSys* sys,
                                const BatchItem* items, const BatchSeg* segs, int nseg, int ctas,
                                long long* grid64, long long gsize, float* rho, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(grid64, 0, sizeof(long long) * gsize, st);
  if (e != cudaSuccess) return e;
  for (int k = 0; k < nseg; k++) {
    const BatchItem* it = items + segs[k].first;
    const int cnt = segs[k].count;
    if (cnt <= 0) continue;
    switch (segs[k].W) {
      case 9: e = batch_scatter_w<9>(sorted, start, sys, it, cnt, ctas, grid64, st); break;
      case 11: e = batch_scatter_w<11>(sorted, start, sys, it, cnt, ctas, grid64, st); break;
      case 13: e = batch_scatter_w<13>(sorted, start, sys, it, cnt, ctas, grid64, st); break;
      case 15: e = batch_scatter_w<15>(sorted, start, sys, it, cnt, ctas, grid64, st); break;
      default: e = cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
  }
  k_grid64_to_real<<<sm_count() * 8, 256, 0, st>>>(grid64, gsize, rho);
  return cudaGetLastError();
}

cudaError_t launch_batch_green(float2* rhok, const float* tab, long long ktot, const BatchSys* sys,
                               const long long* kfirst, const int* ksys, int nsys, double* energy,
                               cudaStream_t st) {
  k_batch_green_apply<<<sm_count() * 8, 256, 0, st>>>(rhok, tab, ktot, sys, kfirst, ksys, nsys, energy);
  return cudaGetLastError();
}

cudaError_t launch_batch_gather(const float4* sorted, const int* perm, const int* start,
                                const BatchSys* sys, const BatchItem* items, const BatchSeg* segs,
                                int nseg, int ctas, const float* phi, double outscale, double* fx,
                                double* fy, double* fz, cudaStream_t st) {
  for (int k = 0; k < nseg; k++) {
    const BatchItem* it = items + segs[k].first;
    const int cnt = segs[k].count;
    if (cnt <= 0) continue;
    cudaError_t e;
    switch (segs[k].W) {
      case 9: e = batch_gather_w<9>(sorted, perm, start, sys, it, cnt, ctas, phi, outscale, fx, fy, fz, st); break;
      case 11: e = batch_gather_w<11>(sorted, perm, start, sys, it, cnt, ctas, phi, outscale, fx, fy, fz, st); break;
      case 13: e = batch_gather_w<13>(sorted, perm, start, sys, it, cnt, ctas, phi, outscale, fx, fy, fz, st); break;
      case 15: e = batch_gather_w<15>(sorted, perm, start, sys, it, cnt, ctas, phi, outscale, fx, fy, fz, st); break;
      default: e = cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}


// ===========================================================================
// Batched systems in one persistent cooperative launch
// ===========================================================================
constexpr int kFusedThreads = 512;
static_assert(kFusedThreads == kScatterThreads, "the fused kernel runs the scatter bricks");
static_assert(kScanTile % kFusedThreads == 0, "scan tile per thread");

constexpr size_t cmax(size_t a, size_t b) { return a > b ? a : b; }

template <int GL>
constexpr size_t fused_fwd_smem() {
  return cmax(cmax(cmax(sizeof(int) * ScatterGeom<9>::words, sizeof(int) * ScatterGeom<11>::words),
                   cmax(sizeof(int) * ScatterGeom<13>::words, sizeof(int) * ScatterGeom<15>::words)),
              cmax(cmax(cmax(GatherGeom<float, 9, kFusedThreads, GL>::bytes,
                             GatherGeom<float, 11, kFusedThreads, GL>::bytes),
                        cmax(GatherGeom<float, 13, kFusedThreads, GL>::bytes,
                             GatherGeom<float, 15, kFusedThreads, GL>::bytes)),
                   sizeof(SmallFftTw) + sizeof(int) * 3 * (kSfSmemSystems + 1)));
}

bool batch_fused_supported(const BatchSys* sys, int nsys) {
  for (int s = 0; s < nsys; s++) {
    for (int d = 0; d < 3; d++)
      if (sys[s].b.M[d] % 8 != 0 || sys[s].b.M[d] > kSfMax) return false;
    if (sys[s].W != 9 && sys[s].W != 11 && sys[s].W != 13 && sys[s].W != 15) return false;
  }
  return nsys > 0;
}

// One tile of kScanTile bin counts: exclusive prefix into start, the tile's
// sum into tile_sums[t].  All threads of the block.
__device__ __forceinline__ int fused_scan_tile(const int* __restrict__ counts, int nb,
                                               int* __restrict__ start, int* __restrict__ sums,
                                               int t) {
  constexpr int PER = kScanTile / kFusedThreads;
  const int base = t * kScanTile + threadIdx.x * PER;
  int v[PER];
  int s = 0;
#pragma unroll
  for (int j = 0; j < PER; j++) {
    v[j] = (base + j < nb) ? counts[base + j] : 0;
    s += v[j];
  }
  int total;
  int run = block_exclusive_scan(s, &total);
#pragma unroll
  for (int j = 0; j < PER; j++) {
    if (base + j < nb) start[base + j] = run;
    run += v[j];
  }
  if (threadIdx.x == 0) sums[t] = total;
  return total;
}

template <int GL>
__global__ void __launch_bounds__(kFusedThreads, 1) k_batch_forward_fused(BatchFused a) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) unsigned char fsm[];
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long gstride = (long long)gridDim.x * blockDim.x;
  // clear the bin counts and the int64 grid
  for (long long i = gtid; i < a.nbins; i += gstride) a.w.counts[i] = 0;
  for (long long i = gtid; i < a.gtot; i += gstride) a.g64[i] = 0;
  if (gtid < 2) a.qctr[gtid] = 0;
  cg::this_grid().sync();
  // bin keys and counts (the key of k_batch_bin_count)
  for (long long i = gtid; i < a.ntot; i += gstride) {
    const float4 p = a.xyzq[i];
    const BatchSys& S = a.sys[batch_sys_of(a.first, a.nsys, (int)i)];
    const int cx = wrap1(centre_cell(p.x, S.sp.inv_h[0]), S.b.M[0]);
    const int cy = wrap1(centre_cell(p.y, S.sp.inv_h[1]), S.b.M[1]);
    const int cz = wrap1(centre_cell(p.z, S.sp.inv_h[2]), S.b.M[2]);
    const int k = S.bin_off + (cz * S.b.M[1] + cy) * S.b.nbx + (cx >> S.b.bxs);
    a.w.key[i] = k;
    atomicAdd(&a.w.counts[k], 1);
  }
  cg::this_grid().sync();
  // exclusive scan of the counts: tiles, their sums, the offsets
  const int ntiles = (a.nbins + kScanTile - 1) / kScanTile;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    fused_scan_tile(a.w.counts, a.nbins, a.w.start, a.w.tile_sums, t);
  cg::this_grid().sync();
  if (blockIdx.x == 0) {  // tile sums -> tile offsets, in place (ntiles <= kScanTile)
    const int total = fused_scan_tile(a.w.tile_sums, ntiles, a.w.tile_sums,
                                      a.w.tile_sums + ntiles, 0);
    if (threadIdx.x == 0) a.w.start[a.nbins] = total;
  }
  cg::this_grid().sync();
  for (long long i = gtid; i < a.nbins; i += gstride) a.w.start[i] += a.w.tile_sums[i / kScanTile];
  cg::this_grid().sync();
  // placement in any order within a bin (the counts return to zero)
  for (long long i = gtid; i < a.ntot; i += gstride) {
    const int k = a.w.key[i];
    const int slot = a.w.start[k] + atomicSub(&a.w.counts[k], 1) - 1;
    a.sorted[slot] = a.xyzq[i];
    a.perm[slot] = (int)i;
  }
  cg::this_grid().sync();
  // spread bricks
  for (int it = fused_next_item(&a.qctr[0]); it < a.nscat; it = fused_next_item(&a.qctr[0])) {
    const BatchItem item = a.scat[it];
    const BatchSys& S = a.sys[item.sys];
    const int* st = a.w.start + S.bin_off;
    long long* g = a.g64 + S.grid_off;
    int* tile = reinterpret_cast<int*>(fsm);
    switch (S.W) {
      case 9: scatter_brick<9>(a.sorted, st, S.b, S.sp, item.bx, item.by, item.bz, tile, g); break;
      case 11: scatter_brick<11>(a.sorted, st, S.b, S.sp, item.bx, item.by, item.bz, tile, g); break;
      case 13: scatter_brick<13>(a.sorted, st, S.b, S.sp, item.bx, item.by, item.bz, tile, g); break;
      default: scatter_brick<15>(a.sorted, st, S.b, S.sp, item.bx, item.by, item.bz, tile, g); break;
    }
    __syncthreads();
  }
  cg::this_grid().sync();
  fused_solve(a, a.phi, true, fsm);
  cg::this_grid().sync();
  // gather bricks
  for (int it = fused_next_item(&a.qctr[1]); it < a.ngath; it = fused_next_item(&a.qctr[1])) {
    const BatchItem item = a.gath[it];
    const BatchSys& S = a.sys[item.sys];
    const int* st = a.w.start + S.bin_off;
    const float* ph = a.phi + S.grid_off;
    switch (S.W) {
      case 9:
        gather_brick<float, 9, kFusedThreads, GL>(a.sorted, a.perm, st, S.b, S.sg, ph, a.ccelec,
                                                  a.fx, a.fy, a.fz, item.bx, item.by, item.bz, fsm);
        break;
      case 11:
        gather_brick<float, 11, kFusedThreads, GL>(a.sorted, a.perm, st, S.b, S.sg, ph, a.ccelec,
                                                   a.fx, a.fy, a.fz, item.bx, item.by, item.bz, fsm);
        break;
      case 13:
        gather_brick<float, 13, kFusedThreads, GL>(a.sorted, a.perm, st, S.b, S.sg, ph, a.ccelec,
                                                   a.fx, a.fy, a.fz, item.bx, item.by, item.bz, fsm);
        break;
      default:
        gather_brick<float, 15, kFusedThreads, GL>(a.sorted, a.perm, st, S.b, S.sg, ph, a.ccelec,
                                                   a.fx, a.fy, a.fz, item.bx, item.by, item.bz, fsm);
        break;
    }
    __syncthreads();
  }
}

template <int GL>
static int fused_fwd_ctas() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return 0;
  }
  int v = cache[dev].load();
  if (v == 0) {
    const size_t smem = fused_fwd_smem<GL>();
    int nb = 0;
    if (cudaFuncSetAttribute(k_batch_forward_fused<GL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_batch_forward_fused<GL>,
                                                      kFusedThreads, smem) != cudaSuccess) {
      cudaGetLastError();
      nb = 0;
    }
    v = nb > 0 ? nb * sm_count() : -1;
    cache[dev].store(v);
  }
  return v > 0 ? v : 0;
}

int batch_fused_ctas(int gather_lanes) {
  return gather_lanes == 8 ? fused_fwd_ctas<8>() : fused_fwd_ctas<16>();
}

cudaError_t launch_batch_forward_fused(const BatchFused& a, int ctas, int gather_lanes,
                                       cudaStream_t st) {
  const int most = gather_lanes == 8 ? fused_fwd_ctas<8>() : fused_fwd_ctas<16>();
  if (most <= 0 || ctas < 1 || ctas > most) return cudaErrorCooperativeLaunchTooLarge;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(kFusedThreads);
  cfg.dynamicSmemBytes = gather_lanes == 8 ? fused_fwd_smem<8>() : fused_fwd_smem<16>();
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (gather_lanes == 8) return cudaLaunchKernelEx(&cfg, k_batch_forward_fused<8>, a);
  return cudaLaunchKernelEx(&cfg, k_batch_forward_fused<16>, a);
}

#define GSE_TILED_INST(CT)                                                                      \
  template cudaError_t launch_bin_sorted<CT>(const Vec4<CT>::type*, int, const BinLayout&, CT,  \
                                             CT, CT, BinScratch, Vec4<CT>::type*, int*,         \
                                             cudaStream_t);                                     \
  template cudaError_t launch_bin_scan_place<CT>(const Vec4<CT>::type*, int, int, BinScratch,   \
                                                 Vec4<CT>::type*, int*, cudaStream_t);          \
  template bool spread_tiled_supported<CT>(const Stencil<CT>&);                                 \
  template cudaError_t launch_spread_tiled<CT>(const Vec4<CT>::type*, const int*,               \
                                               const unsigned*, const BinLayout&,               \
                                               const Stencil<CT>&, CT*, cudaStream_t);          \
  template cudaError_t launch_gather_tiled<CT>(const Vec4<CT>::type*, const int*, const int*,   \
                                               const BinLayout&, const Stencil<CT>&, const CT*, \
                                               double, double*, double*, double*, bool,         \
                                               cudaStream_t);

GSE_TILED_INST(double)
GSE_TILED_INST(float)

}  // namespace gse
