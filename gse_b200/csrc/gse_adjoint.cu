// gse_adjoint.cu -- reverse-mode derivatives of one GSE-k force evaluation.
//
// The forward pass (CpuGSEk::spreadCharge1 -> solvePoisson -> calculateEnergy
// -> interpolateForce, CpuGSEk.cpp:30-58, CpuGSE.cpp:70-103) is
//   rho(r) = sum_i q_i g(r - x_i)          over the (2n+1)^3 cube of atom i,
//            g = (2 pi s^2)^(-3/2) exp(-|r - x|^2 / (2 s^2)), s = sigma1
//   phi    = K rho                          K = c2r G(sigma2) r2c (symmetric)
//   E      = 1/2 c h^3 rho . phi            c = ccelec, h^3 = cell volume
//   F_i    = c q_i sum_{r in sphere_i} D_i(r) phi(r),
//            D_i(r) = A exp(-|u|^2 / (2 s^2)) u,  u = x_i - r,
//            A = (2 pi)^(-3/2) h^3 s^-5.
// Given dL/dE = gE and dL/dF_i = G_i, with
//   lambda(r) = c sum_i q_i G_i . D_i(r)     (the adjoint source, sphere)
//   Psi       = K lambda + gE c h^3 phi      (dL/drho)
// the derivatives are
//   dL/dq_j = sum_{cube} g(r - x_j) Psi(r) + c A sum_{sphere} e phi (G_j . u)
//   dL/dx_j = q_j sum_{cube} g (r - x_j) / s^2 Psi(r)
//           + c q_j A sum_{sphere} e phi [G_j - (G_j . u) u / s^2],
// e = exp(-|u|^2 / (2 s^2)).  The sphere's edge is not differentiated (its
// derivative is zero almost everywhere).
#include "gse_adjoint.cuh"
#include "gse_internal.cuh"
#include "gse_tiled.cuh"

namespace gse {

// lambda(r) += c q_i A e (G_i . u) over the sphere of atom i (global atomics);
// one warp per atom.
template <typename CT>
__device__ __forceinline__ void adj_source_atom(const typename Vec4<CT>::type& a, int i,
                                                const Stencil<CT>& s, double c,
                                                const double* __restrict__ gfx,
                                                const double* __restrict__ gfy,
                                                const double* __restrict__ gfz,
                                                CT* __restrict__ lambda) {
  const int lane = threadIdx.x & 31;
  const int W0 = 2 * s.nst[0] + 1, W1 = 2 * s.nst[1] + 1, W2 = 2 * s.nst[2] + 1;
  {
    const CT pos[3] = {a.x, a.y, a.z};
    const CT G[3] = {(CT)gfx[i], (CT)gfy[i], (CT)gfz[i]};
    const CT amp = (CT)(c * (double)a.w * (double)s.pref);
    int c0[3];
#pragma unroll
    for (int d = 0; d < 3; d++) c0[d] = round_to_int(mul_rn(pos[d], s.inv_h[d])) - s.nst[d];
    for (int t = lane; t < W0 * W1 * W2; t += 32) {
      const int tz = t / (W0 * W1), r = t - tz * W0 * W1, ty = r / W0, tx = r - ty * W0;
      const int p[3] = {c0[0] + tx, c0[1] + ty, c0[2] + tz};
      CT u[3];
#pragma unroll
      for (int d = 0; d < 3; d++) u[d] = sub_rn(pos[d], mul_rn((CT)p[d], s.h[d]));
      const CT r2 = add_rn(add_rn(mul_rn(u[0], u[0]), mul_rn(u[1], u[1])), mul_rn(u[2], u[2]));
      if (r2 < s.rcut2) {
        const CT e = gexp(-r2 * s.inv_2s2);
        const CT v = amp * e * (G[0] * u[0] + G[1] * u[1] + G[2] * u[2]);
        const long long idx = pmod(p[0], s.M[0]) +
                              ((long long)pmod(p[1], s.M[1]) + (long long)pmod(p[2], s.M[2]) * s.M[1]) * s.M[0];
        atomicAdd(lambda + idx, v);
      }
    }
  }
}

template <typename CT>
__global__ void __launch_bounds__(256)
    k_adj_source(const typename Vec4<CT>::type* __restrict__ xyzq, const int* __restrict__ perm,
                 int n, Stencil<CT> s, double c, const double* __restrict__ gfx,
                 const double* __restrict__ gfy, const double* __restrict__ gfz,
                 CT* __restrict__ lambda) {
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int ii = gw; ii < n; ii += nw)
    adj_source_atom<CT>(xyzq[ii], perm[ii], s, c, gfx, gfy, gfz, lambda);
}

// Per atom: the cube gather of Psi = psi + gE c h^3 phi and the sphere
// gather of phi, combined into dL/dq and dL/dx.
template <typename CT>
__device__ __forceinline__ void adj_gather_atom(
    const typename Vec4<CT>::type& a, int i, const Stencil<CT>& sp, const Stencil<CT>& sg,
    double c, double gE_ch3, const CT* __restrict__ psi, const CT* __restrict__ phi,
    const double* __restrict__ gfx, const double* __restrict__ gfy,
    const double* __restrict__ gfz, double* __restrict__ dq, double* __restrict__ dx,
    double* __restrict__ dy, double* __restrict__ dz) {
  const int lane = threadIdx.x & 31;
  const int W0 = 2 * sp.nst[0] + 1, W1 = 2 * sp.nst[1] + 1, W2 = 2 * sp.nst[2] + 1;
  const double inv_s2 = 2.0 * (double)sp.inv_2s2;
  {
    const CT pos[3] = {a.x, a.y, a.z};
    const double G[3] = {gfx ? gfx[i] : 0.0, gfy ? gfy[i] : 0.0, gfz ? gfz[i] : 0.0};
    int c0[3];
#pragma unroll
    for (int d = 0; d < 3; d++) c0[d] = round_to_int(mul_rn(pos[d], sp.inv_h[d])) - sp.nst[d];
    double P = 0, V[3] = {0, 0, 0}, T0 = 0, T1[3] = {0, 0, 0}, T2[3] = {0, 0, 0};
    for (int t = lane; t < W0 * W1 * W2; t += 32) {
      const int tz = t / (W0 * W1), r = t - tz * W0 * W1, ty = r / W0, tx = r - ty * W0;
      const int p[3] = {c0[0] + tx, c0[1] + ty, c0[2] + tz};
      CT u[3];
#pragma unroll
      for (int d = 0; d < 3; d++) u[d] = sub_rn(pos[d], mul_rn((CT)p[d], sp.h[d]));
      const CT r2 = add_rn(add_rn(mul_rn(u[0], u[0]), mul_rn(u[1], u[1])), mul_rn(u[2], u[2]));
      const long long idx = pmod(p[0], sp.M[0]) +
                            ((long long)pmod(p[1], sp.M[1]) + (long long)pmod(p[2], sp.M[2]) * sp.M[1]) * sp.M[0];
      const double e = (double)gexp(-r2 * sp.inv_2s2);
      const double ph = (double)phi[idx];
      const double Psi = (double)psi[idx] + gE_ch3 * ph;
      const double g = (double)sp.pref * e * Psi;  // g(r - x) Psi
      P += g;
#pragma unroll
      for (int d = 0; d < 3; d++) V[d] -= g * (double)u[d] * inv_s2;  // (r - x) = -u
      if (r2 < sg.rcut2) {
        const double t0 = e * ph;
        const double Gu = G[0] * (double)u[0] + G[1] * (double)u[1] + G[2] * (double)u[2];
        T0 += t0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
          T1[d] += t0 * (double)u[d];
          T2[d] += t0 * Gu * (double)u[d];
        }
      }
    }
    P = warp_sum(P);
    T0 = warp_sum(T0);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      V[d] = warp_sum(V[d]);
      T1[d] = warp_sum(T1[d]);
      T2[d] = warp_sum(T2[d]);
    }
    if (lane == 0) {
      const double q = (double)a.w;
      const double cA = c * (double)sg.pref;
      dq[i] = P + cA * (G[0] * T1[0] + G[1] * T1[1] + G[2] * T1[2]);
      dx[i] = q * V[0] + cA * q * (G[0] * T0 - T2[0] * inv_s2);
      dy[i] = q * V[1] + cA * q * (G[1] * T0 - T2[1] * inv_s2);
      dz[i] = q * V[2] + cA * q * (G[2] * T0 - T2[2] * inv_s2);
    }
  }
}

template <typename CT>
__global__ void __launch_bounds__(256)
    k_adj_gather(const typename Vec4<CT>::type* __restrict__ xyzq, const int* __restrict__ perm,
                 int n, Stencil<CT> sp /*spread*/, Stencil<CT> sg /*gather*/, double c,
                 double gE_ch3, const CT* __restrict__ psi, const CT* __restrict__ phi,
                 const double* __restrict__ gfx, const double* __restrict__ gfy,
                 const double* __restrict__ gfz, double* __restrict__ dq,
                 double* __restrict__ dx, double* __restrict__ dy, double* __restrict__ dz) {
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int ii = gw; ii < n; ii += nw)
    adj_gather_atom<CT>(xyzq[ii], perm[ii], sp, sg, c, gE_ch3, psi, phi, gfx, gfy, gfz, dq, dx,
                        dy, dz);
}

// ---- batched systems: system of a sorted atom by its offset range ----
__device__ __forceinline__ int adj_sys_of(const int* __restrict__ first, int nsys, int i) {
  int lo = 0, hi = nsys - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(256)
    k_batch_adj_source(const float4* __restrict__ xyzq, const int* __restrict__ perm, int ntot,
                       const BatchSys* __restrict__ sys, const int* __restrict__ first, int nsys,
                       double c, const double* __restrict__ gfx, const double* __restrict__ gfy,
                       const double* __restrict__ gfz, float* __restrict__ lambda) {
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int ii = gw; ii < ntot; ii += nw) {
    const BatchSys& S = sys[adj_sys_of(first, nsys, ii)];
    adj_source_atom<float>(xyzq[ii], perm[ii], S.sg, c, gfx, gfy, gfz, lambda + S.grid_off);
  }
}

__global__ void __launch_bounds__(256)
    k_batch_adj_gather(const float4* __restrict__ xyzq, const int* __restrict__ perm, int ntot,
                       const BatchSys* __restrict__ sys, const int* __restrict__ first, int nsys,
                       double c, const double* __restrict__ dLdE, const float* __restrict__ psi,
                       const float* __restrict__ phi, const double* __restrict__ gfx,
                       const double* __restrict__ gfy, const double* __restrict__ gfz,
                       double* __restrict__ dq, double* __restrict__ dx, double* __restrict__ dy,
                       double* __restrict__ dz) {
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int ii = gw; ii < ntot; ii += nw) {
    const int si = adj_sys_of(first, nsys, ii);
    const BatchSys& S = sys[si];
    adj_gather_atom<float>(xyzq[ii], perm[ii], S.sp, S.sg, c, dLdE[si] * c * S.h3,
                           psi + S.grid_off, phi + S.grid_off, gfx, gfy, gfz, dq, dx, dy, dz);
  }
}

cudaError_t launch_batch_adj_source(const float4* xyzq, const int* perm, int ntot,
                                    const BatchSys* sys, const int* first, int nsys, double c,
                                    const double* gfx, const double* gfy, const double* gfz,
                                    float* lambda, cudaStream_t st) {
  if (ntot <= 0) return cudaSuccess;
  k_batch_adj_source<<<148 * 16, 256, 0, st>>>(xyzq, perm, ntot, sys, first, nsys, c, gfx, gfy,
                                               gfz, lambda);
  return cudaGetLastError();
}

cudaError_t launch_batch_adj_gather(const float4* xyzq, const int* perm, int ntot,
                                    const BatchSys* sys, const int* first, int nsys, double c,
                                    const double* dLdE, const float* psi, const float* phi,
                                    const double* gfx, const double* gfy, const double* gfz,
                                    double* dq, double* dx, double* dy, double* dz,
                                    cudaStream_t st) {
  if (ntot <= 0) return cudaSuccess;
  k_batch_adj_gather<<<148 * 16, 256, 0, st>>>(xyzq, perm, ntot, sys, first, nsys, c, dLdE, psi,
                                               phi, gfx, gfy, gfz, dq, dx, dy, dz);
  return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_adj_source(const typename Vec4<CT>::type* xyzq, const int* perm, int n,
                              const Stencil<CT>& s, double c, const double* gfx,
                              const double* gfy, const double* gfz, CT* lambda, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int blocks = (int)std::min<long long>(148 * 16, (n + 7) / 8);
  k_adj_source<CT><<<blocks, 256, 0, st>>>(xyzq, perm, n, s, c, gfx, gfy, gfz, lambda);
  return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_adj_gather(const typename Vec4<CT>::type* xyzq, const int* perm, int n,
                              const Stencil<CT>& sp, const Stencil<CT>& sg, double c,
                              double gE_ch3, const CT* psi, const CT* phi, const double* gfx,
                              const double* gfy, const double* gfz, double* dq, double* dx,
                              double* dy, double* dz, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int blocks = (int)std::min<long long>(148 * 16, (n + 7) / 8);
  k_adj_gather<CT><<<blocks, 256, 0, st>>>(xyzq, perm, n, sp, sg, c, gE_ch3, psi, phi, gfx, gfy,
                                           gfz, dq, dx, dy, dz);
  return cudaGetLastError();
}

#define GSE_ADJ_INST(CT)                                                                        \
  template cudaError_t launch_adj_source<CT>(const Vec4<CT>::type*, const int*, int,           \
                                             const Stencil<CT>&, double, const double*,          \
                                             const double*, const double*, CT*, cudaStream_t);   \
  template cudaError_t launch_adj_gather<CT>(const Vec4<CT>::type*, const int*, int,           \
                                             const Stencil<CT>&, const Stencil<CT>&, double,     \
                                             double, const CT*, const CT*, const double*,        \
                                             const double*, const double*, double*, double*,     \
                                             double*, double*, cudaStream_t);

GSE_ADJ_INST(double)
GSE_ADJ_INST(float)

}  // namespace gse
