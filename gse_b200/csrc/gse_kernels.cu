// gse_kernels.cu -- CUDA kernels of the GSE-k path (sm_100a).
//
// Stage map (reference = ap-hynninen/GSE):
//   k_spread_atomic  CpuGaussCharge::spreadChargeToGrid  (CpuGaussCharge.cpp:235-384)
//   k_fixed_to_real  int64 fixed-point grid -> CT grid (mixed form)
//   k_green_energy   CpuGreensFuncGSE::mul (CpuGreensFuncGSE.cpp:9-57) fused with
//                    the mesh energy of CpuGSE::calculateEnergy (CpuGSE.cpp:86-103)
//                    evaluated in k-space (Parseval)
//   k_dot            real-space energy sum, CpuGSE.cpp:96-97
//   k_gather         CpuGaussCharge::interpolateLoop (CpuGaussCharge.cpp:105-172)
#include "gse_internal.cuh"
#include "gse_kernels.cuh"
#include "gse_reduce.cuh"

namespace gse {

// ---------------------------------------------------------------------------
// Spread: one warp per atom.  The three 1-D weight rows are computed once per
// atom, w[j] = exp(-(d0 + j h)^2 / (2 sigma^2)) with d0 = c*h - x and
// c = round(x/h) - n, exactly the reference's separable form
// (CpuGaussCharge.cpp:306-329); each of the (2n+1)^3 cube points adds
// q*pref*wx*wy*wz into the periodic grid.  FIXED accumulates
// round(v * fixed_scale) as int64, which makes the sum independent of the
// order of the atomics.
// ---------------------------------------------------------------------------
template <typename CT, bool FIXED>
__global__ void __launch_bounds__(256)
    k_spread_atomic(const typename Vec4<CT>::type* __restrict__ xyzq, int n, Stencil<CT> s,
                    CT* __restrict__ grid, unsigned long long* __restrict__ fixed_grid) {
  __shared__ CT wsh[8][3][kMaxStencil];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int gw = blockIdx.x * (blockDim.x >> 5) + wib;
  const int nw = gridDim.x * (blockDim.x >> 5);
  const int W0 = 2 * s.nst[0] + 1, W1 = 2 * s.nst[1] + 1, W2 = 2 * s.nst[2] + 1;
  const int W01 = W0 * W1, Wt = W01 * W2;
  CT* w[3] = {wsh[wib][0], wsh[wib][1], wsh[wib][2]};
  const bool wrap_once = (W0 <= s.M[0]) && (W1 <= s.M[1]) && (W2 <= s.M[2]);
  for (int i = gw; i < n; i += nw) {
    const auto a = xyzq[i];
    const CT q_pref = a.w * s.pref;
    const CT pos[3] = {a.x, a.y, a.z};
    int base[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const int c = round_to_int(mul_rn(pos[d], s.inv_h[d])) - s.nst[d];
      const CT d0 = sub_rn(mul_rn((CT)c, s.h[d]), pos[d]);
      const int W = 2 * s.nst[d] + 1;
      for (int j = lane; j < W; j += 32) {
        const CT t = add_rn(d0, mul_rn((CT)j, s.h[d]));
        w[d][j] = gexp(mul_rn(mul_rn(-t, t), s.inv_2s2));
      }
      base[d] = pmod(c, s.M[d]);
    }
    __syncwarp();
    if (s.normalize) {
      // CpuGaussCharge.cpp:330-362: rescale each row to sum sqrt(2 pi sigma^2)
      if (lane < 3) {
        const int W = 2 * (lane == 0 ? s.nst[0] : (lane == 1 ? s.nst[1] : s.nst[2])) + 1;
        CT* wl = wsh[wib][lane];
        CT sum = (CT)0;
        for (int j = 0; j < W; j++) sum += wl[j];
        const CT nrm = s.norm_pref1 / sum;
        for (int j = 0; j < W; j++) wl[j] *= nrm;
      }
      __syncwarp();
    }
    for (int t = lane; t < Wt; t += 32) {
      const int tz = t / W01;
      const int r = t - tz * W01;
      const int ty = r / W0;
      const int tx = r - ty * W0;
      int gx = base[0] + tx, gy = base[1] + ty, gz = base[2] + tz;
      if (wrap_once) {
        gx -= (gx >= s.M[0]) ? s.M[0] : 0;
        gy -= (gy >= s.M[1]) ? s.M[1] : 0;
        gz -= (gz >= s.M[2]) ? s.M[2] : 0;
      } else {
        gx %= s.M[0];
        gy %= s.M[1];
        gz %= s.M[2];
      }
      const long long idx = gx + ((long long)gy + (long long)gz * s.M[1]) * s.M[0];
      const CT v = q_pref * w[0][tx] * w[1][ty] * w[2][tz];
      if (FIXED) {
        const long long iv = llrint((double)v * s.fixed_scale);
        atomicAdd(fixed_grid + idx, (unsigned long long)iv);
      } else {
        atomicAdd(grid + idx, v);
      }
    }
    __syncwarp();
  }
}

template <typename CT>
__global__ void k_fixed_to_real(const long long* __restrict__ in, long long size,
                                double inv_scale, CT* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < size;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (CT)((double)in[i] * inv_scale);
}

// Green's-function multiply on the r2c half spectrum [nz][ny][nx/2+1],
// CpuGreensFuncGSE.cpp:28-56, with the energy sum_k G |rho(k)|^2 over the
// full spectrum (the half-spectrum bins kx = 1 .. ceil(nx/2)-1 stand for two
// bins each).  The FP64 form evaluates G in the reference's order and type;
// the mixed form evaluates G in FP64 and rounds it to FP32.
template <typename CT>
__global__ void __launch_bounds__(256)
    k_green_energy(typename Cplx<CT>::type* __restrict__ rhok, GreenGeom g,
                   double* __restrict__ partials) {
  const long long total = (long long)g.sizeX * g.nfft[1] * g.nfft[2];
  double e = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    auto v = rhok[idx];
    if (idx == 0) {
      v.x = (CT)0;
      v.y = (CT)0;
      rhok[0] = v;
      continue;
    }
    const int ix = (int)(idx % g.sizeX);
    const long long r = idx / g.sizeX;
    const int iy = (int)(r % g.nfft[1]);
    const int iz = (int)(r / g.nfft[1]);
    const int kx = (ix >= g.half[0]) ? ix - g.nfft[0] : ix;
    const int ky = (iy >= g.half[1]) ? iy - g.nfft[1] : iy;
    const int kz = (iz >= g.half[2]) ? iz - g.nfft[2] : iz;
    const double kxd = (double)kx * g.twopi_box[0];
    const double kyd = (double)ky * g.twopi_box[1];
    const double kzd = (double)kz * g.twopi_box[2];
    const double kd2 = add_rn(add_rn(mul_rn(kxd, kxd), mul_rn(kyd, kyd)), mul_rn(kzd, kzd));
    const double facd = g.fourpi_vol * exp(-g.sigmafac * kd2) / kd2;
    const CT fac = (CT)facd;
    if (g.want_energy) {
      const double wgt = (ix == 0 || (g.nx_even && ix == g.nfft[0] / 2)) ? 1.0 : 2.0;
      const double re = (double)v.x, im = (double)v.y;
      e += wgt * (double)fac * (re * re + im * im);
    }
    v.x *= fac;
    v.y *= fac;
    rhok[idx] = v;
  }
  if (g.want_energy) block_sum_to(e, partials);
}

// G(k) of CpuGreensFuncGSE.cpp:28-56 evaluated once in FP64 for every bin of
// the half spectrum and stored in CT (0 at k = 0).
template <typename CT>
__global__ void k_green_table(GreenGeom g, CT* __restrict__ tab) {
  const long long total = (long long)g.sizeX * g.nfft[1] * g.nfft[2];
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    if (idx == 0) {
      tab[0] = (CT)0;
      continue;
    }
    const int ix = (int)(idx % g.sizeX);
    const long long r = idx / g.sizeX;
    const int iy = (int)(r % g.nfft[1]);
    const int iz = (int)(r / g.nfft[1]);
    const int kx = (ix >= g.half[0]) ? ix - g.nfft[0] : ix;
    const int ky = (iy >= g.half[1]) ? iy - g.nfft[1] : iy;
    const int kz = (iz >= g.half[2]) ? iz - g.nfft[2] : iz;
    const double kxd = (double)kx * g.twopi_box[0];
    const double kyd = (double)ky * g.twopi_box[1];
    const double kzd = (double)kz * g.twopi_box[2];
    const double kd2 = add_rn(add_rn(mul_rn(kxd, kxd), mul_rn(kyd, kyd)), mul_rn(kzd, kzd));
    tab[idx] = (CT)(g.fourpi_vol * exp(-g.sigmafac * kd2) / kd2);
  }
}

// rhok *= G (table) with the energy sum_k G |rho(k)|^2 over the full
// spectrum: every bin counts twice except kx = 0 and the kx Nyquist bin.
// The energy is finished in the kernel by its last block (last_block_sum).
template <typename CT>
__global__ void __launch_bounds__(256)
    k_green_apply(typename Cplx<CT>::type* __restrict__ rhok, const CT* __restrict__ tab,
                  GreenGeom g, double* __restrict__ partials, double factor,
                  double* __restrict__ energy_out) {
  const unsigned total = (unsigned)g.sizeX * g.nfft[1] * g.nfft[2];
  const unsigned sx = (unsigned)g.sizeX;
  const unsigned nyq = g.nx_even ? (unsigned)(g.nfft[0] / 2) : 0xffffffffu;
  double e = 0.0;
  auto bin = [&](typename Cplx<CT>::type& v, CT f, unsigned ix) {
    const double re = (double)v.x, im = (double)v.y;
    const double wgt = (ix == 0 || ix == nyq) ? 1.0 : 2.0;
    e += wgt * (double)f * (re * re + im * im);
    v.x *= f;
    v.y *= f;
  };
  if constexpr (sizeof(CT) == 4) {
    // two bins per thread and step: one 16-byte load of rho(k), one 8-byte
    // load of G (cudaMalloc'd buffers, even bin index)
    const unsigned pairs = total / 2;
    float4* r4 = reinterpret_cast<float4*>(rhok);
    const float2* t2 = reinterpret_cast<const float2*>(tab);
    for (unsigned j = blockIdx.x * blockDim.x + threadIdx.x; j < pairs;
         j += gridDim.x * blockDim.x) {
      float4 w = r4[j];
      const float2 f = t2[j];
      const unsigned ix0 = (2 * j) % sx, ix1 = ix0 + 1 == sx ? 0 : ix0 + 1;
      float2 a = make_float2(w.x, w.y), b = make_float2(w.z, w.w);
      bin(a, f.x, ix0);
      bin(b, f.y, ix1);
      r4[j] = make_float4(a.x, a.y, b.x, b.y);
    }
    if ((total & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
      auto v = rhok[total - 1];
      bin(v, tab[total - 1], (total - 1) % sx);
      rhok[total - 1] = v;
    }
  } else {
    for (unsigned idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += gridDim.x * blockDim.x) {
      auto v = rhok[idx];
      bin(v, tab[idx], idx % sx);
      rhok[idx] = v;
    }
  }
  block_sum_to(e, partials);
  last_block_sum(partials, factor, energy_out);
}

// Reciprocal-space virial from the half spectrum rho^ and the Green's table:
// with E_k = factor w_k G(k) |rho^(k)|^2 (w_k = 1 on the x' = 0 and Nyquist
// planes, 2 elsewhere; sum_k E_k is the mesh energy),
//   W_ab = sum_k E_k (delta_ab - 2 k_a k_b (1/k^2 + sigma^2/2)),
// sigma the total Gaussian width (the spread's sigma1 enters |rho^|^2 twice,
// the Green's function sigma2 once: sigma^2 = 2 sigma1^2 + sigma2^2).
// Components xx, yy, zz, xy, xz, yz into out[0..5]; block sums to
// partials[c * gridDim.x + block], the last block adds them in index order.
template <typename CT>
__global__ void __launch_bounds__(256)
    k_virial(const typename Cplx<CT>::type* __restrict__ rhok, const CT* __restrict__ tab,
             GreenGeom g, double half_sigma2, double factor, double* __restrict__ partials,
             unsigned* __restrict__ done, double* __restrict__ out) {
  const unsigned total = (unsigned)g.sizeX * g.nfft[1] * g.nfft[2];
  const unsigned nyq = g.nx_even ? (unsigned)(g.nfft[0] / 2) : 0xffffffffu;
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (unsigned idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += gridDim.x * blockDim.x) {
    const unsigned ix = idx % (unsigned)g.sizeX, t = idx / (unsigned)g.sizeX;
    const int iy = (int)(t % (unsigned)g.nfft[1]), iz = (int)(t / (unsigned)g.nfft[1]);
    const double kx = g.twopi_box[0] * (double)ix;
    const double ky = g.twopi_box[1] * (double)(iy >= g.half[1] ? iy - g.nfft[1] : iy);
    const double kz = g.twopi_box[2] * (double)(iz >= g.half[2] ? iz - g.nfft[2] : iz);
    const double k2 = kx * kx + ky * ky + kz * kz;
    if (k2 == 0.0) continue;
    const auto r = rhok[idx];
    const double re = (double)r.x, im = (double)r.y;
    const double e = ((ix == 0 || ix == nyq) ? 1.0 : 2.0) * (double)tab[idx] * (re * re + im * im);
    const double c = 2.0 * (1.0 / k2 + half_sigma2);
    v[0] += e * (1.0 - c * kx * kx);
    v[1] += e * (1.0 - c * ky * ky);
    v[2] += e * (1.0 - c * kz * kz);
    v[3] -= e * c * kx * ky;
    v[4] -= e * c * kx * kz;
    v[5] -= e * c * ky * kz;
  }
  __shared__ double red[6][32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int d = 0; d < 6; d++) {
    const double s = warp_sum(v[d]);
    if (lane == 0) red[d][wid] = s;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int d = 0; d < 6; d++) {
      const double s = warp_sum(lane < nw ? red[d][lane] : 0.0);
      if (lane == 0) partials[d * gridDim.x + blockIdx.x] = s;
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
  for (int d = 0; d < 6; d++) {
    double t = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
      t += ((volatile double*)partials)[d * gridDim.x + i];
    t = warp_sum(t);
    if (lane == 0) red[d][wid] = t;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int d = 0; d < 6; d++) {
      const double t = warp_sum(lane < nw ? red[d][lane] : 0.0);
      if (lane == 0) out[d] = t * factor;
    }
    if (lane == 0) *done = 0u;
  }
}

template <typename CT>
cudaError_t launch_virial(const typename Cplx<CT>::type* rhok, const CT* tab, const GreenGeom& g,
                          double half_sigma2, double factor, double* partials, unsigned* done,
                          int nblocks, double* out, cudaStream_t st) {
  k_virial<CT><<<nblocks, 256, 0, st>>>(rhok, tab, g, half_sigma2, factor, partials, done, out);
  return cudaGetLastError();
}
template cudaError_t launch_virial<double>(const double2*, const double*, const GreenGeom&, double,
                                           double, double*, unsigned*, int, double*, cudaStream_t);
template cudaError_t launch_virial<float>(const float2*, const float*, const GreenGeom&, double,
                                          double, double*, unsigned*, int, double*, cudaStream_t);

// Copy of the atoms with every charge set to 1 (the field at the atoms is
// the gather of a unit charge); in and out may be the same buffer.
template <typename CT>
__global__ void k_unit_charges(const typename Vec4<CT>::type* in, typename Vec4<CT>::type* out,
                               int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    typename Vec4<CT>::type a = in[i];
    a.w = (CT)1;
    out[i] = a;
  }
}

template <typename CT>
cudaError_t launch_unit_charges(const typename Vec4<CT>::type* in, typename Vec4<CT>::type* out,
                                int n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_unit_charges<CT><<<std::min((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(in, out, n);
  return cudaGetLastError();
}
template cudaError_t launch_unit_charges<double>(const double4*, double4*, int, cudaStream_t);
template cudaError_t launch_unit_charges<float>(const float4*, float4*, int, cudaStream_t);

// factor * sum_i (double)(a[i]*b[i]) (the product in CT, as CpuGSE.cpp:97),
// finished by the last block.  done is the zeroed counter the last block
// resets (the slot after the partials that the other energy kernels use).
template <typename CT>
__global__ void __launch_bounds__(256)
    k_dot(const CT* __restrict__ a, const CT* __restrict__ b, long long size,
          double* __restrict__ partials, unsigned* __restrict__ done, double factor,
          double* __restrict__ out) {
  // four independent partial sums, each step's loads issued together
  double e[4] = {0.0, 0.0, 0.0, 0.0};
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if constexpr (sizeof(CT) == 4) {
    // four points per 16-byte load (cudaMalloc'd grids), four loads per step
    const long long quads = size / 4;
    const float4* a4 = reinterpret_cast<const float4*>(a);
    const float4* b4 = reinterpret_cast<const float4*>(b);
    for (long long i = t0; i < quads; i += 4 * stride) {
      float4 u[4], v[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const long long j = i + k * stride;
        if (j < quads) {
          u[k] = a4[j];
          v[k] = b4[j];
        } else {
          u[k] = v[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
#pragma unroll
      for (int k = 0; k < 4; k++) {
        e[k] += (double)(u[k].x * v[k].x);
        e[k] += (double)(u[k].y * v[k].y);
        e[k] += (double)(u[k].z * v[k].z);
        e[k] += (double)(u[k].w * v[k].w);
      }
    }
    if (blockIdx.x == 0)
      for (long long i = quads * 4 + threadIdx.x; i < size; i += blockDim.x)
        e[0] += (double)(a[i] * b[i]);
  } else {
    const long long pairs = size / 2;
    const double2* a2 = reinterpret_cast<const double2*>(a);
    const double2* b2 = reinterpret_cast<const double2*>(b);
    for (long long i = t0; i < pairs; i += 4 * stride) {
      double2 u[4], v[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const long long j = i + k * stride;
        if (j < pairs) {
          u[k] = a2[j];
          v[k] = b2[j];
        } else {
          u[k] = v[k] = make_double2(0.0, 0.0);
        }
      }
#pragma unroll
      for (int k = 0; k < 4; k++) {
        e[k] += u[k].x * v[k].x;
        e[k] += u[k].y * v[k].y;
      }
    }
    if (blockIdx.x == 0)
      for (long long i = pairs * 2 + threadIdx.x; i < size; i += blockDim.x) e[0] += a[i] * b[i];
  }
  block_sum_to((e[0] + e[1]) + (e[2] + e[3]), partials);
  last_block_sum_counter(partials, done, factor, out);
}

__global__ void k_energy_finalize(const double* __restrict__ partials, int np, double factor,
                                  double* __restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += partials[i];
  s = warp_sum(s);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = s;
  __syncthreads();
  if (w == 0) {
    double t = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) out[0] = t * factor;
  }
}

// ---------------------------------------------------------------------------
// Gather: one warp per atom, lanes over the (ty, tz) rows of the stencil, each
// lane walking its row along x.  The spherical cut is evaluated exactly as
// the reference does, r2 = (dx*dx + dy*dy) + dz*dz in CT with separately
// rounded operations (CpuGaussCharge.cpp:145-158); the Gaussian factor is the
// product of the 1-D factors exp(-dx^2/(2 sigma^2)) exp(-dy^2..) exp(-dz^2..).
// Output: res = outscale * q * pref * sum w phi (x - x_p), written (not
// accumulated) to the atom's original index.
// ---------------------------------------------------------------------------
template <typename CT, typename ACC>
__global__ void __launch_bounds__(256)
    k_gather(const typename Vec4<CT>::type* __restrict__ xyzq, const int* __restrict__ perm,
             int n, Stencil<CT> s, const CT* __restrict__ phi, double outscale,
             double* __restrict__ fx, double* __restrict__ fy, double* __restrict__ fz) {
  __shared__ CT tab[8][3][3][kMaxStencil];   // [warp][axis][d, d^2, w][j]
  __shared__ int off[8][3][kMaxStencil];     // wrapped index * axis stride
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int gw = blockIdx.x * (blockDim.x >> 5) + wib;
  const int nw = gridDim.x * (blockDim.x >> 5);
  const int W0 = 2 * s.nst[0] + 1, W1 = 2 * s.nst[1] + 1, W2 = 2 * s.nst[2] + 1;
  const int stride[3] = {1, s.M[0], s.M[0] * s.M[1]};
  for (int ii = gw; ii < n; ii += nw) {
    const auto a = xyzq[ii];
    const CT fac = a.w * s.pref;
    const CT pos[3] = {a.x, a.y, a.z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const int c = round_to_int(mul_rn(pos[d], s.inv_h[d]));
      const int W = 2 * s.nst[d] + 1;
      for (int j = lane; j < W; j += 32) {
        const int t = c - s.nst[d] + j;
        const CT dd = sub_rn(pos[d], mul_rn((CT)t, s.h[d]));
        const CT d2 = mul_rn(dd, dd);
        tab[wib][d][0][j] = dd;
        tab[wib][d][1][j] = d2;
        tab[wib][d][2][j] = gexp(mul_rn(-d2, s.inv_2s2));
        off[wib][d][j] = pmod(t, s.M[d]) * stride[d];
      }
    }
    __syncwarp();
    ACC ax = 0, ay = 0, az = 0;
    for (int row = lane; row < W1 * W2; row += 32) {
      const int tz = row / W1;
      const int ty = row - tz * W1;
      const CT dy2 = tab[wib][1][1][ty], dz2 = tab[wib][2][1][tz];
      if (!(add_rn(dy2, dz2) < s.rcut2)) continue;  // whole row outside the sphere
      const CT* prow = phi + off[wib][1][ty] + off[wib][2][tz];
      CT s0 = (CT)0, s1 = (CT)0;
      for (int k = 0; k < W0; k++) {
        const CT r2 = add_rn(add_rn(tab[wib][0][1][k], dy2), dz2);
        if (r2 < s.rcut2) {
          const CT wph = tab[wib][0][2][k] * __ldg(prow + off[wib][0][k]);
          s0 += wph;
          s1 += wph * tab[wib][0][0][k];
        }
      }
      const CT wyz = tab[wib][1][2][ty] * tab[wib][2][2][tz];
      ax += (ACC)(wyz * s1);
      ay += (ACC)(wyz * tab[wib][1][0][ty] * s0);
      az += (ACC)(wyz * tab[wib][2][0][tz] * s0);
    }
    ax = warp_sum(ax);
    ay = warp_sum(ay);
    az = warp_sum(az);
    if (lane == 0) {
      const int o = perm ? perm[ii] : ii;
      const double f = outscale * (double)fac;
      fx[o] = f * (double)ax;
      fy[o] = f * (double)ay;
      fz[o] = f * (double)az;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Host-side launchers
// ---------------------------------------------------------------------------
static int blocks_for(long long work, int per_block, int cap) {
  long long b = (work + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

template <typename CT>
cudaError_t launch_spread(const typename Vec4<CT>::type* xyzq, int n, const Stencil<CT>& s,
                          CT* grid, long long* fixed_grid, cudaStream_t st) {
  const long long size = (long long)s.M[0] * s.M[1] * s.M[2];
  cudaError_t e;
  if (fixed_grid)
    e = cudaMemsetAsync(fixed_grid, 0, sizeof(long long) * size, st);
  else
    e = cudaMemsetAsync(grid, 0, sizeof(CT) * size, st);
  if (e != cudaSuccess) return e;
  if (n > 0) {
    const int gb = blocks_for(n, 8, sm_count() * 16);
    if (fixed_grid)
      k_spread_atomic<CT, true><<<gb, 256, 0, st>>>(xyzq, n, s, grid,
                                                    (unsigned long long*)fixed_grid);
    else
      k_spread_atomic<CT, false><<<gb, 256, 0, st>>>(xyzq, n, s, grid, nullptr);
  }
  if (fixed_grid) {
    k_fixed_to_real<CT><<<blocks_for(size, 256, sm_count() * 16), 256, 0, st>>>(
        fixed_grid, size, 1.0 / s.fixed_scale, grid);
  }
  return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_green_energy(typename Cplx<CT>::type* rhok, const GreenGeom& g,
                                double* partials, int np, double factor, double* energy_out,
                                cudaStream_t st) {
  k_green_energy<CT><<<np, 256, 0, st>>>(rhok, g, partials);
  if (g.want_energy) k_energy_finalize<<<1, 1024, 0, st>>>(partials, np, factor, energy_out);
  return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_green_table(const GreenGeom& g, CT* tab, cudaStream_t st) {
  k_green_table<CT><<<sm_count() * 8, 256, 0, st>>>(g, tab);
  return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_green_apply(typename Cplx<CT>::type* rhok, const CT* tab, const GreenGeom& g,
                               double* partials, int np, double factor, double* energy_out,
                               cudaStream_t st) {
  k_green_apply<CT><<<np, 256, 0, st>>>(rhok, tab, g, partials, factor, energy_out);
  return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_dot_energy(const CT* a, const CT* b, long long size, double* partials, int np,
                              double factor, double* energy_out, cudaStream_t st) {
  // fewer, fuller blocks than the other energy kernels; the counter stays in
  // the slot after np partials that they use
  k_dot<CT><<<std::min(np, sm_count() * 4), 256, 0, st>>>(
      a, b, size, partials, reinterpret_cast<unsigned*>(partials + np), factor, energy_out);
  return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_gather(const typename Vec4<CT>::type* xyzq, const int* perm, int n,
                          const Stencil<CT>& s, const CT* phi, double outscale, double* fx,
                          double* fy, double* fz, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int gb = blocks_for(n, 8, sm_count() * 16);
  typedef typename std::conditional<sizeof(CT) == 8, double, float>::type ACC;
  k_gather<CT, ACC><<<gb, 256, 0, st>>>(xyzq, perm, n, s, phi, outscale, fx, fy, fz);
  return cudaGetLastError();
}

#define GSE_INSTANTIATE(CT)                                                                    \
  template cudaError_t launch_spread<CT>(const Vec4<CT>::type*, int, const Stencil<CT>&, CT*,  \
                                         long long*, cudaStream_t);                            \
  template cudaError_t launch_green_energy<CT>(Cplx<CT>::type*, const GreenGeom&, double*,     \
                                               int, double, double*, cudaStream_t);            \
  template cudaError_t launch_green_table<CT>(const GreenGeom&, CT*, cudaStream_t);             \
  template cudaError_t launch_green_apply<CT>(Cplx<CT>::type*, const CT*, const GreenGeom&,     \
                                              double*, int, double, double*, cudaStream_t);     \
  template cudaError_t launch_dot_energy<CT>(const CT*, const CT*, long long, double*, int,    \
                                             double, double*, cudaStream_t);                   \
  template cudaError_t launch_gather<CT>(const Vec4<CT>::type*, const int*, int,               \
                                         const Stencil<CT>&, const CT*, double, double*,       \
                                         double*, double*, cudaStream_t);

GSE_INSTANTIATE(double)
GSE_INSTANTIATE(float)

}  // namespace gse
