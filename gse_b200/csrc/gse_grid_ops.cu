// gse_grid_ops.cu -- grid-to-grid operations of CpuGaussCharge beside the
// force path, for both calculation types:
//
//   k_conv_x,     the periodic 1-D passes of the on-grid Gaussian convolution
//   k_conv_yz     (spreadChargeOnGrid, CpuGaussCharge.cpp:390-519); three
//                 passes x -> y -> z make the convolution, the z taps carry
//                 the prefactor
//   k_efield      the forward-difference electric field on the grid
//                 (calcElectricFieldOnGrid, CpuGaussCharge.cpp:62-98)
//   k_dipole      the dipole sum of a charge grid (calcDipoleSum,
//                 CpuGaussCharge.cpp:188-226)
//
// All three stream whole grids with the warps' loads and stores along x.  The
// convolution passes stage a run of input with its halo in shared memory by
// independent loads (many lines in flight per thread), then sum the taps
// from there; the field takes one warp per x row, the dipole one CTA per row.  The
// arithmetic is the reference's, operation for operation, with explicit
// round-to-nearest intrinsics so that no multiply-add is contracted: the
// convolution and the field are bit-identical to the reference, the dipole
// terms too (their sum is a fixed-order tree instead of the reference's loop
// order).
#include "gse_grid_ops.cuh"

namespace gse {

namespace {

// p + d wrapped into [0, m) for any d (the taps may be wider than the grid)
__device__ __forceinline__ int wrap_any(int v, int m) {
  if ((unsigned)v < (unsigned)m) return v;
  v %= m;
  return v < 0 ? v + m : v;
}

}  // namespace

// x pass: each warp takes a run of at most kConvRunX outputs of one row; the
// run and its 2n-point halo are read into shared memory by independent
// coalesced loads (several per lane in flight), then each lane sums the taps
// of its outputs from there.
constexpr int kConvRunX = 160;
// y and z passes: a CTA of 32 x 8 threads takes 32 x-columns by kConvRun
// outputs along the axis; the kConvRun + 2n rows it needs are staged first.
constexpr int kConvRun = 72;

template <typename CT>
__global__ void __launch_bounds__(256)
    k_conv_x(const CT* __restrict__ in, CT* __restrict__ out, int mx, long long rows, int run,
             ConvTaps<CT> taps) {
  __shared__ CT g[kMaxStencil];
  __shared__ CT buf[8][kConvRunX + kMaxStencil];
  const int n = taps.n, w = 2 * n + 1;
  const int lane = threadIdx.x, wp = threadIdx.y;
  for (int i = wp * 32 + lane; i < w; i += 256) g[i] = taps.g[i];
  __syncthreads();
  const long long r = (long long)blockIdx.x * 8 + wp;
  if (r >= rows) return;
  const int x0 = blockIdx.y * run;
  const int len = min(run, mx - x0);
  if (len <= 0) return;
  const CT* row = in + r * mx;
  CT* b = buf[wp];
  for (int i = lane; i < len + 2 * n; i += 32) b[i] = row[wrap_any(x0 - n + i, mx)];
  __syncwarp();
  for (int i = lane; i < len; i += 32) {
    CT s = (CT)0;
    for (int t = 0; t < w; t++) s = add_rn(s, mul_rn(g[t], b[i + t]));
    out[r * mx + x0 + i] = s;
  }
}

// axis 1 (y, stride mx) or 2 (z, stride mx*my); blockIdx.z runs over the
// remaining axis (z for the y pass, y for the z pass).
template <typename CT>
__global__ void __launch_bounds__(256)
    k_conv_yz(const CT* __restrict__ in, CT* __restrict__ out, int mx, int my, int mz, int axis,
              int run, ConvTaps<CT> taps) {
  __shared__ CT g[kMaxStencil];
  __shared__ CT buf[kConvRun + kMaxStencil][33];
  const int n = taps.n, w = 2 * n + 1;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  for (int i = tid; i < w; i += 256) g[i] = taps.g[i];
  const int ma = axis == 1 ? my : mz;
  const long long stride = axis == 1 ? (long long)mx : (long long)mx * my;
  const long long ostride = axis == 1 ? (long long)mx * my : (long long)mx;
  const int x = blockIdx.x * 32 + tx;
  const int a0 = blockIdx.y * run;
  const int len = min(run, ma - a0);
  const CT* base = in + (long long)blockIdx.z * ostride + x;
  if (x < mx)
    for (int i = ty; i < len + 2 * n; i += 8)
      buf[i][tx] = base[(long long)wrap_any(a0 - n + i, ma) * stride];
  __syncthreads();
  if (x >= mx) return;
  CT* obase = out + (long long)blockIdx.z * ostride + x;
  for (int i = ty; i < len; i += 8) {
    CT s = (CT)0;
    for (int t = 0; t < w; t++) s = add_rn(s, mul_rn(g[t], buf[i + t][tx]));
    obase[(long long)(a0 + i) * stride] = s;
  }
}

// The same two passes for a tap count W known at compile time: the taps sit
// in registers, the tap loops unroll and each thread issues all of its loads
// before it stores any of them to shared memory, so that they are in flight
// together.  The y/z kernel gives each thread kConvK consecutive outputs, one
// window of kConvK + W - 1 staged values in registers feeding kConvK
// independent sums; in the x kernel each warp takes one row run and each
// lane the outputs lane, lane + 32, ...
constexpr int kConvK = 9;
static_assert(kConvK * 8 == kConvRun, "8 rows of threads cover one run");

template <typename CT, int W>
__global__ void __launch_bounds__(256)
    k_conv_x_w(const CT* __restrict__ in, CT* __restrict__ out, int mx, long long rows, int run,
               ConvTaps<CT> taps) {
  constexpr int n = (W - 1) / 2;
  constexpr int NL = (kConvRunX + W - 1 + 31) / 32;
  __shared__ CT buf[8][kConvRunX + W];
  CT g[W];
#pragma unroll
  for (int t = 0; t < W; t++) g[t] = taps.g[t];
  const int lane = threadIdx.x, wp = threadIdx.y;
  const long long r = (long long)blockIdx.x * 8 + wp;
  if (r >= rows) return;
  const int x0 = blockIdx.y * run;
  const int len = min(run, mx - x0);
  if (len <= 0) return;
  const CT* row = in + r * mx;
  CT* b = buf[wp];
  CT ld[NL];
#pragma unroll
  for (int k = 0; k < NL; k++) {
    const int i = lane + 32 * k;
    ld[k] = i < len + 2 * n ? row[wrap_any(x0 - n + i, mx)] : (CT)0;
  }
#pragma unroll
  for (int k = 0; k < NL; k++) {
    const int i = lane + 32 * k;
    if (i < len + 2 * n) b[i] = ld[k];
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < kConvRunX / 32; k++) {
    const int i = lane + 32 * k;
    if (i < len) {
      CT s = (CT)0;
#pragma unroll
      for (int t = 0; t < W; t++) s = add_rn(s, mul_rn(g[t], b[i + t]));
      out[r * mx + x0 + i] = s;
    }
  }
}

template <typename CT, int W>
__global__ void __launch_bounds__(256)
    k_conv_yz_w(const CT* __restrict__ in, CT* __restrict__ out, int mx, int my, int mz,
                int axis, int run, ConvTaps<CT> taps) {
  constexpr int n = (W - 1) / 2;
  constexpr int NL = (kConvRun + W - 1 + 7) / 8;
  __shared__ CT buf[kConvRun + W - 1][33];
  CT g[W];
#pragma unroll
  for (int t = 0; t < W; t++) g[t] = taps.g[t];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int ma = axis == 1 ? my : mz;
  const long long stride = axis == 1 ? (long long)mx : (long long)mx * my;
  const long long ostride = axis == 1 ? (long long)mx * my : (long long)mx;
  const int x = blockIdx.x * 32 + tx;
  const int a0 = blockIdx.y * run;
  const int len = min(run, ma - a0);
  const CT* base = in + (long long)blockIdx.z * ostride + x;
  if (x < mx) {
    CT ld[NL];
#pragma unroll
    for (int k = 0; k < NL; k++) {
      const int i = ty + 8 * k;
      ld[k] = i < len + 2 * n ? base[(long long)wrap_any(a0 - n + i, ma) * stride] : (CT)0;
    }
#pragma unroll
    for (int k = 0; k < NL; k++) {
      const int i = ty + 8 * k;
      if (i < len + 2 * n) buf[i][tx] = ld[k];
    }
  }
  __syncthreads();
  const int i0 = ty * kConvK;
  if (x >= mx || i0 >= len) return;
  // rows past len + 2n were not staged; they feed only outputs past len
  CT v[kConvK + W - 1];
#pragma unroll
  for (int j = 0; j < kConvK + W - 1; j++) v[j] = i0 + j < len + 2 * n ? buf[i0 + j][tx] : (CT)0;
  CT* obase = out + (long long)blockIdx.z * ostride + x;
#pragma unroll
  for (int k = 0; k < kConvK; k++) {
    if (i0 + k < len) {
      CT s = (CT)0;
#pragma unroll
      for (int t = 0; t < W; t++) s = add_rn(s, mul_rn(g[t], v[k + t]));
      obase[(long long)(a0 + i0 + k) * stride] = s;
    }
  }
}

template <typename CT>
__global__ void __launch_bounds__(256)
    k_efield(const CT* __restrict__ phi, CT* __restrict__ ex, CT* __restrict__ ey,
             CT* __restrict__ ez, int mx, int my, int mz, CT ihx, CT ihy, CT ihz) {
  const long long rows = (long long)my * mz;
  const long long plane = (long long)mx * my;
  const long long r = (long long)blockIdx.x * 8 + threadIdx.y;  // one row per warp
  if (r >= rows) return;
  const int y = (int)(r % my), z = (int)(r / my);
  const long long ry = (long long)(y + 1 == my ? 0 : y + 1) * mx + (long long)z * plane;
  const long long rz = (long long)y * mx + (long long)(z + 1 == mz ? 0 : z + 1) * plane;
  // four x positions per lane and step, their loads issued together
  for (int xb = 0; xb < mx; xb += 128) {
    CT c[4], px[4], py[4], pz[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int x = xb + threadIdx.x + 32 * k;
      if (x < mx) {
        c[k] = phi[r * mx + x];
        px[k] = phi[r * mx + (x + 1 == mx ? 0 : x + 1)];
        py[k] = phi[ry + x];
        pz[k] = phi[rz + x];
      }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int x = xb + threadIdx.x + 32 * k;
      if (x < mx) {
        const long long p = r * mx + x;
        ex[p] = mul_rn(-sub_rn(px[k], c[k]), ihx);
        ey[p] = mul_rn(-sub_rn(py[k], c[k]), ihy);
        ez[p] = mul_rn(-sub_rn(pz[k], c[k]), ihz);
      }
    }
  }
}

template <typename CT>
__global__ void __launch_bounds__(256)
    k_dipole(const CT* __restrict__ rho, int mx, int my, int mz, CT hx, CT hy, CT hz,
             double* __restrict__ partials, unsigned* __restrict__ done,
             double* __restrict__ out) {
  const long long rows = (long long)my * mz;
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    const int y = (int)(r % my), z = (int)(r / my);
    const CT cy = mul_rn(hy, (CT)y), cz = mul_rn(hz, (CT)z);
    for (int x = threadIdx.x; x < mx; x += blockDim.x) {
      const CT val = mul_rn(mul_rn(mul_rn(rho[r * mx + x], hx), hy), hz);
      sx += (double)mul_rn(val, mul_rn(hx, (CT)x));
      sy += (double)mul_rn(val, cy);
      sz += (double)mul_rn(val, cz);
    }
  }
  // block sums in a fixed tree, then the last block adds the block sums in
  // index order: the result does not depend on which block ran when
  __shared__ double red[3][32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double v[3] = {sx, sy, sz};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    v[d] = warp_sum(v[d]);
    if (lane == 0) red[d][wid] = v[d];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double t = lane < nw ? red[d][lane] : 0.0;
      t = warp_sum(t);
      if (lane == 0) partials[d * gridDim.x + blockIdx.x] = t;
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double t = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
      t += ((volatile double*)partials)[d * gridDim.x + i];
    t = warp_sum(t);
    if (lane == 0) red[d][wid] = t;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double t = lane < nw ? red[d][lane] : 0.0;
      t = warp_sum(t);
      if (lane == 0) out[d] = t;
    }
    if (lane == 0) *done = 0u;
  }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
template <typename CT>
cudaError_t launch_conv_pass(const CT* in, CT* out, const int M[3], int axis,
                             const ConvTaps<CT>& taps, cudaStream_t st) {
  if (taps.n < 0 || 2 * taps.n + 1 > kMaxStencil || axis < 0 || axis > 2)
    return cudaErrorInvalidValue;
  const int W = 2 * taps.n + 1;
  const dim3 blk(32, 8);
  if (axis == 0) {
    const long long rows = (long long)M[1] * M[2];
    const int nruns = (M[0] + kConvRunX - 1) / kConvRunX;
    const int run = (M[0] + nruns - 1) / nruns;
    const long long groups = (rows + 7) / 8;
    if (groups > 0x7fffffffLL || nruns > 65535) return cudaErrorInvalidValue;
    const dim3 grid((unsigned)groups, nruns);
    switch (W) {
#define CONV_X(WW) \
  case WW:         \
    k_conv_x_w<CT, WW><<<grid, blk, 0, st>>>(in, out, M[0], rows, run, taps); \
    break;
      CONV_X(5) CONV_X(7) CONV_X(9) CONV_X(11) CONV_X(13) CONV_X(15)
#undef CONV_X
      default:
        k_conv_x<CT><<<grid, blk, 0, st>>>(in, out, M[0], rows, run, taps);
    }
  } else {
    const int ma = axis == 1 ? M[1] : M[2], other = axis == 1 ? M[2] : M[1];
    const int nruns = (ma + kConvRun - 1) / kConvRun;
    const int run = (ma + nruns - 1) / nruns;
    if (other > 65535 || nruns > 65535) return cudaErrorInvalidValue;
    const dim3 grid((M[0] + 31) / 32, nruns, other);
    switch (W) {
#define CONV_YZ(WW) \
  case WW:          \
    k_conv_yz_w<CT, WW><<<grid, blk, 0, st>>>(in, out, M[0], M[1], M[2], axis, run, taps); \
    break;
      CONV_YZ(5) CONV_YZ(7) CONV_YZ(9) CONV_YZ(11) CONV_YZ(13) CONV_YZ(15)
#undef CONV_YZ
      default:
        k_conv_yz<CT><<<grid, blk, 0, st>>>(in, out, M[0], M[1], M[2], axis, run, taps);
    }
  }
  return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_efield(const CT* phi, CT* ex, CT* ey, CT* ez, const int M[3],
                          const CT inv_h[3], cudaStream_t st) {
  const long long groups = ((long long)M[1] * M[2] + 7) / 8;
  if (groups > 0x7fffffffLL) return cudaErrorInvalidValue;
  k_efield<CT><<<(unsigned)groups, dim3(32, 8), 0, st>>>(phi, ex, ey, ez, M[0], M[1], M[2],
                                                          inv_h[0], inv_h[1], inv_h[2]);
  return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_dipole(const CT* rho, const int M[3], const CT h[3], double* partials,
                          unsigned* done, double* out, cudaStream_t st) {
  const long long rows = (long long)M[1] * M[2];
  const int nb = (int)std::min<long long>(rows, std::min(kDipoleBlocks, sm_count() * 4));
  k_dipole<CT><<<nb, 256, 0, st>>>(rho, M[0], M[1], M[2], h[0], h[1], h[2], partials, done, out);
  return cudaGetLastError();
}

#define INSTANTIATE(CT)                                                                        \
  template cudaError_t launch_conv_pass<CT>(const CT*, CT*, const int[3], int,                 \
                                            const ConvTaps<CT>&, cudaStream_t);                \
  template cudaError_t launch_efield<CT>(const CT*, CT*, CT*, CT*, const int[3], const CT[3],  \
                                         cudaStream_t);                                        \
  template cudaError_t launch_dipole<CT>(const CT*, const int[3], const CT[3], double*,        \
                                         unsigned*, double*, cudaStream_t);
INSTANTIATE(double)
INSTANTIATE(float)
#undef INSTANTIATE

}  // namespace gse
