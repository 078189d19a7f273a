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
#include <atomic>
#include <type_traits>

#include "gse_adjoint.cuh"
#include "gse_internal.cuh"
#include "gse_tiled.cuh"
#include "gse_tiled_dev.cuh"

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

// ===========================================================================
// Tiled reverse pass (mixed form)
// ===========================================================================
// The same brick decomposition as the forward pass.  The adjoint source is
// scattered like the charge spread (one warp per atom, lanes over (x, z)
// pairs of the stencil plane, the y values in registers) into an int32 brick
// tile that is added into an int64 grid, so lambda is bit-identical from run
// to run.  The weight of a point is e (G . u) over the gather sphere:
// separable in its y factor, e_x e_z (Gx u_x + Gz u_z) e_y + e_x e_z Gy (e_y u_y).
// The sphere test here is u_y^2 < rcut^2 - (u_x^2 + u_z^2); it may differ
// from the forward gather's association of the same sum only for points
// whose distance equals the cut-off to rounding, whose weight is e^-9 of the
// centre's.

// Per-warp slots for the y tables of the reverse-pass scatter, one array for
// every stencil width a kernel instantiates (a static array in the templated
// function would be one per width, too much static shared memory for the
// fused reverse kernel).
__device__ __forceinline__ float (*adj_ytab())[3][16] {
  __shared__ __align__(16) float t[kScatterThreads / 32][3][16];
  return t;
}

template <int W>
__device__ __forceinline__ void adj_scatter_brick(
    const float4* __restrict__ sorted, const int* __restrict__ perm, const int* __restrict__ start,
    const BinLayout& b, const Stencil<float>& s, float cA, const double* __restrict__ gfx,
    const double* __restrict__ gfy, const double* __restrict__ gfz, int bxi, int byi, int bzi,
    int* __restrict__ tile, long long* __restrict__ grid64) {
  typedef ScatterGeom<W> G;
  constexpr int n = G::n;
  constexpr int NT = kScatterThreads, NW = NT / 32;
  constexpr int NPASS = (W * W + 31) / 32;
  __shared__ int rng_a[kSB * kSB], rng_p[kSB * kSB];
  __shared__ int alist[kScatterList];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int x0 = bxi * kSB, y0 = byi * kSB, z0 = bzi * kSB;
  // |cA q e (G.u)| <= |cA q| |G| max_u |u| exp(-u^2/(2 s^2)) = |cA q| |G| s e^(-1/2)
  const float acA = fabsf(cA) * sqrtf(0.5f / s.inv_2s2) * 0.60653066f * 1.0001f;
  int total;
  const int shift = brick_prologue<W, NT>(
      start, b, x0, y0, z0, tile, rng_a, rng_p,
      [&](int i) {
        const int o = perm[i];
        const float gx = (float)gfx[o], gy = (float)gfy[o], gz = (float)gfz[o];
        return fabsf(sorted[i].w) * acA * sqrtf(gx * gx + gy * gy + gz * gz);
      },
      &total);
  const float tscale = exp2f((float)shift);
  // (x, z) pairs of the stencil plane each lane tests, the same for every atom
  int psx[NPASS], psz[NPASS];
#pragma unroll
  for (int pass = 0; pass < NPASS; pass++) {
    const int p = pass * 32 + lane;
    psz[pass] = p < W * W ? p / W : 0;
    psx[pass] = p < W * W ? p - (p / W) * W : 0;
  }
  // per warp: the pairs whose column meets the sphere, packed x | z << 4
  __shared__ unsigned char plist_all[NW][W * W];
  float (*ytab)[3][16] = adj_ytab();  // e, u, u^2 along y of each warp's atom
  unsigned char* plist = plist_all[warp];
  for (int c0 = 0; c0 < total; c0 += kScatterList) {
    brick_atom_list<NT, kSB * kSB>(rng_a, rng_p, total, c0, kScatterList, alist);
    __syncthreads();
    const int nc = min(kScatterList, total - c0);
    for (int q = warp; q < nc; q += NW) {
      const int ai = alist[q];
      const float4 a = sorted[ai];
      const int o = perm[ai];
      const float Gx = (float)gfx[o], Gy = (float)gfy[o], Gz = (float)gfz[o];
      const float pos3[3] = {a.x, a.y, a.z};
      const int org[3] = {x0, y0, z0};
      int loc[3];
      float ul[3], u2l[3], el[3];  // lane j < W: u = x - r_j, u^2 and e along each axis
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const int cc = centre_cell(pos3[d], s.inv_h[d]);
        loc[d] = wrap1(cc, s.M[d]) - org[d];
        const float u = sub_rn(pos3[d], mul_rn((float)(cc - n + lane), s.h[d]));
        const float u2 = mul_rn(u, u);
        ul[d] = u;
        u2l[d] = u2;
        el[d] = (lane < W) ? expf(mul_rn(-u2, s.inv_2s2)) : 0.f;
      }
      // the y tables every lane needs, through the warp's shared slots and
      // 16-byte broadcast loads rather than 39 shuffles (as in the spread)
      float ey[W], eyuy[W], uy2[W];
      {
        __syncwarp();  // the warp's previous atom has read its tables
        if (lane < 16) {
          ytab[warp][0][lane] = el[1];
          ytab[warp][1][lane] = ul[1];
          ytab[warp][2][lane] = u2l[1];
        }
        __syncwarp();
        float uy[W];
        const float4* v0 = reinterpret_cast<const float4*>(ytab[warp][0]);
        const float4* v1 = reinterpret_cast<const float4*>(ytab[warp][1]);
        const float4* v2 = reinterpret_cast<const float4*>(ytab[warp][2]);
#pragma unroll
        for (int q4 = 0; q4 < (W + 3) / 4; q4++) {
          const float4 a = v0[q4], b = v1[q4], c = v2[q4];
          const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w},
                      cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (4 * q4 + j < W) {
              ey[4 * q4 + j] = av[j];
              uy[4 * q4 + j] = bv[j];
              uy2[4 * q4 + j] = cv[j];
            }
        }
#pragma unroll
        for (int k = 0; k < W; k++) eyuy[k] = ey[k] * uy[k];
      }
      // the same weights in pairs of y points for the packed fma
      unsigned long long ey2[W / 2], eyuy2[W / 2], magic2;
#pragma unroll
      for (int k = 0; k + 1 < W; k += 2) {
        asm("mov.b64 %0, {%1, %2};" : "=l"(ey2[k / 2]) : "f"(ey[k]), "f"(ey[k + 1]));
        asm("mov.b64 %0, {%1, %2};" : "=l"(eyuy2[k / 2]) : "f"(eyuy[k]), "f"(eyuy[k + 1]));
      }
      asm("mov.b64 %0, {%1, %1};" : "=l"(magic2) : "f"(12582912.0f));
      // compact the (x, z) pairs with u_x^2 + u_z^2 < rcut^2: every point of
      // the other columns lies outside the sphere
      int npair = 0;
#pragma unroll
      for (int pass = 0; pass < NPASS; pass++) {
        const float ux2 = __shfl_sync(0xffffffffu, u2l[0], psx[pass]);
        const float uz2 = __shfl_sync(0xffffffffu, u2l[2], psz[pass]);
        const bool ne = pass * 32 + lane < W * W && ux2 + uz2 < s.rcut2;
        const unsigned m = __ballot_sync(0xffffffffu, ne);
        if (ne) plist[npair + __popc(m & ((1u << lane) - 1u))] =
            (unsigned char)(psx[pass] | (psz[pass] << 4));
        npair += __popc(m);
      }
      __syncwarp();
      const float amp = cA * a.w * tscale;
      int* base = tile + loc[2] * G::PP + loc[1] * G::RP + loc[0];
      for (int i0 = 0; i0 < npair; i0 += 32) {
        const bool live = i0 + lane < npair;
        const int pp = live ? plist[i0 + lane] : 0;
        const int px = pp & 15, pz = pp >> 4;
        const float ex = __shfl_sync(0xffffffffu, el[0], px);
        const float ux = __shfl_sync(0xffffffffu, ul[0], px);
        const float ux2 = __shfl_sync(0xffffffffu, u2l[0], px);
        const float ez = __shfl_sync(0xffffffffu, el[2], pz);
        const float uz = __shfl_sync(0xffffffffu, ul[2], pz);
        const float uz2 = __shfl_sync(0xffffffffu, u2l[2], pz);
        if (live) {
          const float w = amp * ex * ez;
          const float t1 = w * (Gx * ux + Gz * uz), t2 = w * Gy;
          const float rem = s.rcut2 - (ux2 + uz2);
          int* cell = base + pz * G::PP + px;
          unsigned long long t1p, t2p;
          asm("mov.b64 %0, {%1, %1};" : "=l"(t1p) : "f"(t1));
          asm("mov.b64 %0, {%1, %1};" : "=l"(t2p) : "f"(t2));
#pragma unroll
          for (int k = 0; k + 1 < W; k += 2) {
            // |t1 e_y + t2 e_y u_y| < 2^22: both roundings stay at unit spacing;
            // two y points per packed fma, each half rounded as fmaf rounds
            unsigned long long r2;
            asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r2) : "l"(t2p), "l"(eyuy2[k / 2]), "l"(magic2));
            asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(r2) : "l"(t1p), "l"(ey2[k / 2]));
            unsigned lo, hi;
            asm("mov.b64 {%0, %1}, %2;" : "=r"(lo), "=r"(hi) : "l"(r2));
            if (uy2[k] < rem) atomicAdd(cell + k * G::RP, (int)lo - 0x4B400000);
            if (uy2[k + 1] < rem) atomicAdd(cell + (k + 1) * G::RP, (int)hi - 0x4B400000);
          }
          if (uy2[W - 1] < rem) {
            const int v = __float_as_int(fmaf(t1, ey[W - 1], fmaf(t2, eyuy[W - 1], 12582912.0f))) -
                          0x4B400000;
            atomicAdd(cell + (W - 1) * G::RP, v);
          }
        }
      }
      __syncwarp();
    }
    __syncthreads();
  }
  brick_flush<W, NT>(tile, b, x0, y0, z0, shift, grid64);
}

// Shared memory of the reverse-pass gather for stencil width W and a block of
// NT threads.
template <int W, int NT = kAdjThreads>
struct AdjGatherGeom {
  static constexpr int n = (W - 1) / 2;
  static constexpr int TX = kAX + 2 * n, TY = kAY + 2 * n, TZ = kAZ + 2 * n;
  static constexpr int TP = TX | 1;
  static constexpr int ZP = ((TY * TP + 31) / 32) * 32 + ((W * TP) % 32);
  static constexpr int NW = NT / 32;
  static constexpr int APW = 32 / kAdjLanes;  // atoms per warp at a time
  static constexpr size_t bytes =
      sizeof(float) * (2 * TZ * ZP + NW * APW * 9 * kWPad) + sizeof(int) * NW * APW * W * W;
};

// Reverse-pass gather of the atoms of one kAX x kAY x kAZ brick: Psi = psi +
// gE c h^3 phi and phi of the brick plus halo in shared memory; kAdjLanes
// lanes per atom: the cube rows of Psi (moments e, e u_x) and the sphere rows
// of phi (moments e, e u_x, e u_x^2), combined into dL/dq and dL/dx.
template <int W, int NT = kAdjThreads>
__device__ __forceinline__ void adj_gather_brick(
    const float4* __restrict__ sorted, const int* __restrict__ perm, const int* __restrict__ start,
    const BinLayout& b, const Stencil<float>& sp, const Stencil<float>& sg, double c,
    double gE_ch3, const float* __restrict__ psi, const float* __restrict__ phi,
    const double* __restrict__ gfx, const double* __restrict__ gfy,
    const double* __restrict__ gfz, double* __restrict__ dq, double* __restrict__ dx,
    double* __restrict__ dy, double* __restrict__ dz, int bxi, int byi, int bzi,
    unsigned char* smem) {
  typedef AdjGatherGeom<W, NT> AG;
  constexpr int n = AG::n, TX = AG::TX, TY = AG::TY, TZ = AG::TZ, TP = AG::TP, ZP = AG::ZP;
  constexpr int NW = AG::NW, APW = AG::APW, GL = kAdjLanes;
  constexpr int NR = kAY * kAZ;
  constexpr int NG = (W * W + GL - 1) / GL;
  float* tpsi = (float*)smem;                        // [TZ][ZP]
  float* tphi = tpsi + TZ * ZP;                      // [TZ][ZP]
  float* tabs = tphi + TZ * ZP;                      // [NW][APW][axis][u, u^2, e][kWPad]
  int* rowl = (int*)(tabs + NW * APW * 9 * kWPad);   // [NW][APW][W*W]
  __shared__ int rng_a[NR], rng_p[NR + 1];
  __shared__ int alist[kGatherList];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grp = lane / GL, gl = lane % GL;
  const int x0 = bxi * kAX, y0 = byi * kAY, z0 = bzi * kAZ;
  const int ex = min(kAX, b.M[0] - x0), ey = min(kAY, b.M[1] - y0), ez = min(kAZ, b.M[2] - z0);
  int cnt = 0;
  if (tid < NR) {
    const int yy = tid % kAY, zz = tid / kAY;
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
  if (natoms == 0) return;  // uniform
  stage_tile_async<float, TX, TY, TZ, TP, ZP, NW>(psi, b, x0, y0, z0, n, tpsi);
  stage_tile_async<float, TX, TY, TZ, TP, ZP, NW>(phi, b, x0, y0, z0, n, tphi);
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  {
    const float g = (float)gE_ch3;
    for (int i = tid; i < TZ * ZP; i += NT) tpsi[i] = fmaf(g, tphi[i], tpsi[i]);
  }
  __syncthreads();

  float* tb = tabs + (warp * APW + grp) * 9 * kWPad;
  int* rl = rowl + (warp * APW + grp) * W * W;
  int gjy[NG], gjz[NG];
#pragma unroll
  for (int g = 0; g < NG; g++) {
    const int r = g * GL + gl;
    gjz[g] = r < W * W ? r / W : 0;
    gjy[g] = r < W * W ? r - (r / W) * W : 0;
  }
  const unsigned gmask = GL == 32 ? 0xffffffffu : ((1u << GL) - 1u);
  const double pref_sp = (double)sp.pref, inv_s2 = 2.0 * (double)sp.inv_2s2;
  const double cA = c * (double)sg.pref;
  for (int c0 = 0; c0 < natoms; c0 += kGatherList) {
    brick_atom_list<NT, NR>(rng_a, rng_p, natoms, c0, kGatherList, alist);
    __syncthreads();
    const int nc = min(kGatherList, natoms - c0);
    for (int q0 = APW * warp; q0 < nc; q0 += APW * NW) {
      const int q = q0 + grp;
      const bool valid = q < nc;
      const int ai = alist[valid ? q : q0];
      const float4 a = sorted[ai];
      const float pos3[3] = {a.x, a.y, a.z};
      const int org[3] = {x0, y0, z0};
      int loc[3];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const int cc = centre_cell(pos3[d], sp.inv_h[d]);
        loc[d] = wrap1(cc, sp.M[d]) - org[d];
        for (int j = gl; j < W; j += GL) {
          const float u = sub_rn(pos3[d], mul_rn((float)(cc - n + j), sp.h[d]));
          const float u2 = mul_rn(u, u);
          tb[(d * 3 + 0) * kWPad + j] = u;
          tb[(d * 3 + 1) * kWPad + j] = u2;
          tb[(d * 3 + 2) * kWPad + j] = expf(mul_rn(-u2, sp.inv_2s2));
        }
      }
      __syncwarp();
      unsigned long long w2[W];  // (e_x, e_x u_x) per x offset
#pragma unroll
      for (int k = 0; k < W; k++) {
        const float e = tb[(0 * 3 + 2) * kWPad + k];
        const float eu = e * tb[(0 * 3 + 0) * kWPad + k];
        asm("mov.b64 %0, {%1, %2};" : "=l"(w2[k]) : "f"(e), "f"(eu));
      }
      // cube rows of Psi: P = sum e Psi, V = sum e Psi u (a lane's rows summed in
      // FP32, the lanes' sums in FP64 below)
      float P = 0.f, Vx = 0.f, Vy = 0.f, Vz = 0.f;
#pragma unroll
      for (int g = 0; g < NG; g++) {
        if (g * GL + gl < W * W) {
          const int jy = gjy[g], jz = gjz[g];
          const float* row = tpsi + (loc[2] + jz) * ZP + (loc[1] + jy) * TP + loc[0];
          unsigned long long acc = 0ull;
#pragma unroll
          for (int k = 0; k < W; k++) {
            unsigned long long p2;
            asm("mov.b64 %0, {%1, %1};" : "=l"(p2) : "f"(row[k]));
            asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(w2[k]), "l"(p2));
          }
          float r0, r1;
          asm("mov.b64 {%0, %1}, %2;" : "=f"(r0), "=f"(r1) : "l"(acc));
          const float w = tb[(1 * 3 + 2) * kWPad + jy] * tb[(2 * 3 + 2) * kWPad + jz];
          const float a0 = w * r0;
          P += a0;
          Vx += w * r1;
          Vy += a0 * tb[(1 * 3 + 0) * kWPad + jy];
          Vz += a0 * tb[(2 * 3 + 0) * kWPad + jz];
        }
      }
      // sphere rows of phi
      int nrow = 0;
#pragma unroll
      for (int g = 0; g < NG; g++) {
        const int r = g * GL + gl;
        bool ne = false;
        if (r < W * W)
          ne = add_rn(tb[(1 * 3 + 1) * kWPad + gjy[g]], tb[(2 * 3 + 1) * kWPad + gjz[g]]) <
               sg.rcut2;
        const unsigned m = (__ballot_sync(0xffffffffu, ne) >> (GL * grp)) & gmask;
        if (ne) rl[nrow + __popc(m & ((1u << gl) - 1u))] = (gjz[g] << 8) | gjy[g];
        nrow += __popc(m);
      }
      __syncwarp();
      float dx2[W], ex[W], eux[W], eu2[W];
#pragma unroll
      for (int k = 0; k < W; k++) {
        dx2[k] = tb[(0 * 3 + 1) * kWPad + k];
        asm("mov.b64 {%0, %1}, %2;" : "=f"(ex[k]), "=f"(eux[k]) : "l"(w2[k]));
        eu2[k] = ex[k] * dx2[k];
      }
      float T0 = 0, T1x = 0, T1y = 0, T1z = 0;
      float Mxx = 0, Mxy = 0, Mxz = 0, Myy = 0, Myz = 0, Mzz = 0;
      // the end points lie outside the sphere for every row when dx^2 >= rcut^2
      // there (rem <= rcut^2): the rows are then summed over the inner points
      const bool ends = dx2[0] < sg.rcut2 || dx2[W - 1] < sg.rcut2;
      const bool trim = !__any_sync(0xffffffffu, ends);
      for (int i = gl; i < nrow; i += GL) {
        const int r = rl[i];
        const int jz = r >> 8, jy = r & 255;
        const float uy2 = tb[(1 * 3 + 1) * kWPad + jy], uz2 = tb[(2 * 3 + 1) * kWPad + jz];
        const float rem = sg.rcut2 - (uy2 + uz2);
        const float* row = tphi + (loc[2] + jz) * ZP + (loc[1] + jy) * TP + loc[0];
        float s0 = 0.f, s1 = 0.f, s2 = 0.f;
        auto pts = [&](auto tr) {
          constexpr int K0 = decltype(tr)::value ? 1 : 0;
          constexpr int K1 = decltype(tr)::value ? W - 1 : W;
#pragma unroll
          for (int k = K0; k < K1; k++) {
            const float ph = row[k];
            if (dx2[k] < rem) {  // the test guards the fmas; a skipped point adds nothing
              s0 = fmaf(ex[k], ph, s0);
              s1 = fmaf(eux[k], ph, s1);
              s2 = fmaf(eu2[k], ph, s2);
            }
          }
        };
        if (trim)
          pts(std::true_type());
        else
          pts(std::false_type());
        const float w = tb[(1 * 3 + 2) * kWPad + jy] * tb[(2 * 3 + 2) * kWPad + jz];
        const float uy = tb[(1 * 3 + 0) * kWPad + jy], uz = tb[(2 * 3 + 0) * kWPad + jz];
        const float a0 = w * s0, a1 = w * s1;
        T0 += a0;
        T1x += a1;
        T1y += a0 * uy;
        T1z += a0 * uz;
        Mxx += w * s2;
        Mxy += a1 * uy;
        Mxz += a1 * uz;
        Myy += a0 * uy2;
        Myz += a0 * uy * uz;
        Mzz += a0 * uz2;
      }
      double acc14[14] = {P, Vx, Vy, Vz, T0, T1x, T1y, T1z, Mxx, Mxy, Mxz, Myy, Myz, Mzz};
#pragma unroll
      for (int o = GL / 2; o > 0; o >>= 1)
#pragma unroll
        for (int v = 0; v < 14; v++) acc14[v] += __shfl_xor_sync(0xffffffffu, acc14[v], o);
      if (gl == 0 && valid) {
        const int o = perm[ai];
        const double q = (double)a.w;
        const double Gx = gfx ? gfx[o] : 0.0, Gy = gfy ? gfy[o] : 0.0, Gz = gfz ? gfz[o] : 0.0;
        const double T2x = acc14[8] * Gx + acc14[9] * Gy + acc14[10] * Gz;
        const double T2y = acc14[9] * Gx + acc14[11] * Gy + acc14[12] * Gz;
        const double T2z = acc14[10] * Gx + acc14[12] * Gy + acc14[13] * Gz;
        const double vs = -pref_sp * inv_s2;  // (r - x) = -u
        dq[o] = pref_sp * acc14[0] + cA * (Gx * acc14[5] + Gy * acc14[6] + Gz * acc14[7]);
        dx[o] = q * vs * acc14[1] + cA * q * (Gx * acc14[4] - T2x * inv_s2);
        dy[o] = q * vs * acc14[2] + cA * q * (Gy * acc14[4] - T2y * inv_s2);
        dz[o] = q * vs * acc14[3] + cA * q * (Gz * acc14[4] - T2z * inv_s2);
      }
      __syncwarp();
    }
    __syncthreads();
  }
}

template <int W>
__global__ void __launch_bounds__(kScatterThreads)
    k_adj_scatter(const float4* __restrict__ sorted, const int* __restrict__ perm,
                  const int* __restrict__ start, BinLayout b, Stencil<float> s, float cA,
                  const double* __restrict__ gfx, const double* __restrict__ gfy,
                  const double* __restrict__ gfz, long long* __restrict__ grid64) {
  extern __shared__ int atile[];
  adj_scatter_brick<W>(sorted, perm, start, b, s, cA, gfx, gfy, gfz, blockIdx.x, blockIdx.y,
                       blockIdx.z, atile, grid64);
}

template <int W>
__global__ void __launch_bounds__(kAdjThreads, 2)
    k_adj_gather_tiled(const float4* __restrict__ sorted, const int* __restrict__ perm,
                       const int* __restrict__ start, BinLayout b, Stencil<float> sp,
                       Stencil<float> sg, double c, double gE_ch3, const float* __restrict__ psi,
                       const float* __restrict__ phi, const double* __restrict__ gfx,
                       const double* __restrict__ gfy, const double* __restrict__ gfz,
                       double* __restrict__ dq, double* __restrict__ dx, double* __restrict__ dy,
                       double* __restrict__ dz) {
  extern __shared__ __align__(16) unsigned char asm_[];
  adj_gather_brick<W>(sorted, perm, start, b, sp, sg, c, gE_ch3, psi, phi, gfx, gfy, gfz, dq, dx,
                      dy, dz, blockIdx.x, blockIdx.y, blockIdx.z, asm_);
}

template <int W>
__global__ void __launch_bounds__(kScatterThreads)
    k_batch_adj_scatter(const float4* __restrict__ sorted, const int* __restrict__ perm,
                        const int* __restrict__ start, const BatchSys* __restrict__ sys,
                        const BatchItem* __restrict__ items, int nitems, double c,
                        const double* __restrict__ gfx, const double* __restrict__ gfy,
                        const double* __restrict__ gfz, long long* __restrict__ grid64) {
  extern __shared__ int atile[];
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BatchItem item = items[it];
    const BatchSys& S = sys[item.sys];
    const float cA = (float)(c * (double)S.sg.pref);
    adj_scatter_brick<W>(sorted, perm, start + S.bin_off, S.b, S.sg, cA, gfx, gfy, gfz, item.bx,
                         item.by, item.bz, atile, grid64 + S.grid_off);
    __syncthreads();
  }
}

template <int W>
__global__ void __launch_bounds__(kAdjThreads, 2)
    k_batch_adj_gather_tiled(const float4* __restrict__ sorted, const int* __restrict__ perm,
                             const int* __restrict__ start, const BatchSys* __restrict__ sys,
                             const BatchItem* __restrict__ items, int nitems, double c,
                             const double* __restrict__ dLdE, const float* __restrict__ psi,
                             const float* __restrict__ phi, const double* __restrict__ gfx,
                             const double* __restrict__ gfy, const double* __restrict__ gfz,
                             double* __restrict__ dq, double* __restrict__ dx,
                             double* __restrict__ dy, double* __restrict__ dz) {
  extern __shared__ __align__(16) unsigned char asm_[];
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BatchItem item = items[it];
    const BatchSys& S = sys[item.sys];
    const double gE_ch3 = dLdE[item.sys] * c * S.h3;
    adj_gather_brick<W>(sorted, perm, start + S.bin_off, S.b, S.sp, S.sg, c, gE_ch3,
                        psi + S.grid_off, phi + S.grid_off, gfx, gfy, gfz, dq, dx, dy, dz, item.bx,
                        item.by, item.bz, asm_);
    __syncthreads();
  }
}

namespace {
template <class K>
cudaError_t set_smem_once(K kernel, size_t bytes, std::atomic<bool>* done) {
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
cudaError_t adj_scatter_w(const float4* sorted, const int* perm, const int* start,
                          const BinLayout& b, const Stencil<float>& s, double c, const double* gfx,
                          const double* gfy, const double* gfz, long long* grid64, float* lambda,
                          cudaStream_t st) {
  static std::atomic<bool> done[64];
  const size_t smem = sizeof(int) * ScatterGeom<W>::words;
  cudaError_t e = set_smem_once(k_adj_scatter<W>, smem, done);
  if (e != cudaSuccess) return e;
  const long long size = (long long)b.M[0] * b.M[1] * b.M[2];
  e = cudaMemsetAsync(grid64, 0, sizeof(long long) * size, st);
  if (e != cudaSuccess) return e;
  const dim3 grd((b.M[0] + kSB - 1) / kSB, (b.M[1] + kSB - 1) / kSB, (b.M[2] + kSB - 1) / kSB);
  k_adj_scatter<W><<<grd, kScatterThreads, smem, st>>>(sorted, perm, start, b, s,
                                                       (float)(c * (double)s.pref), gfx, gfy, gfz,
                                                       grid64);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_grid64_to_real(grid64, size, lambda, st);
}

template <int W>
cudaError_t adj_gather_w(const float4* sorted, const int* perm, const int* start,
                         const BinLayout& b, const Stencil<float>& sp, const Stencil<float>& sg,
                         double c, double gE_ch3, const float* psi, const float* phi,
                         const double* gfx, const double* gfy, const double* gfz, double* dq,
                         double* dx, double* dy, double* dz, cudaStream_t st) {
  static std::atomic<bool> done[64];
  const size_t smem = AdjGatherGeom<W>::bytes;
  const cudaError_t e = set_smem_once(k_adj_gather_tiled<W>, smem, done);
  if (e != cudaSuccess) return e;
  const dim3 grd((b.M[0] + kAX - 1) / kAX, (b.M[1] + kAY - 1) / kAY, (b.M[2] + kAZ - 1) / kAZ);
  k_adj_gather_tiled<W><<<grd, kAdjThreads, smem, st>>>(sorted, perm, start, b, sp, sg, c, gE_ch3,
                                                        psi, phi, gfx, gfy, gfz, dq, dx, dy, dz);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_adj_scatter(const float4* sorted, const int* perm, const int* start,
                               const BinLayout& b, const Stencil<float>& sg, double c,
                               const double* gfx, const double* gfy, const double* gfz,
                               long long* grid64, float* lambda, cudaStream_t st) {
  switch (2 * sg.nst[0] + 1) {
    case 9: return adj_scatter_w<9>(sorted, perm, start, b, sg, c, gfx, gfy, gfz, grid64, lambda, st);
    case 11: return adj_scatter_w<11>(sorted, perm, start, b, sg, c, gfx, gfy, gfz, grid64, lambda, st);
    case 13: return adj_scatter_w<13>(sorted, perm, start, b, sg, c, gfx, gfy, gfz, grid64, lambda, st);
    case 15: return adj_scatter_w<15>(sorted, perm, start, b, sg, c, gfx, gfy, gfz, grid64, lambda, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_adj_gather_tiled(const float4* sorted, const int* perm, const int* start,
                                    const BinLayout& b, const Stencil<float>& sp,
                                    const Stencil<float>& sg, double c, double gE_ch3,
                                    const float* psi, const float* phi, const double* gfx,
                                    const double* gfy, const double* gfz, double* dq, double* dx,
                                    double* dy, double* dz, cudaStream_t st) {
  switch (2 * sp.nst[0] + 1) {
    case 9: return adj_gather_w<9>(sorted, perm, start, b, sp, sg, c, gE_ch3, psi, phi, gfx, gfy, gfz, dq, dx, dy, dz, st);
    case 11: return adj_gather_w<11>(sorted, perm, start, b, sp, sg, c, gE_ch3, psi, phi, gfx, gfy, gfz, dq, dx, dy, dz, st);
    case 13: return adj_gather_w<13>(sorted, perm, start, b, sp, sg, c, gE_ch3, psi, phi, gfx, gfy, gfz, dq, dx, dy, dz, st);
    case 15: return adj_gather_w<15>(sorted, perm, start, b, sp, sg, c, gE_ch3, psi, phi, gfx, gfy, gfz, dq, dx, dy, dz, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_batch_adj_scatter(const float4* sorted, const int* perm, const int* start,
                                     const BatchSys* sys, const BatchItem* items,
                                     const BatchSeg* segs, int nseg, int ctas, double c,
                                     const double* gfx, const double* gfy, const double* gfz,
                                     long long* grid64, long long gsize, float* lambda,
                                     cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(grid64, 0, sizeof(long long) * gsize, st);
  if (e != cudaSuccess) return e;
  for (int k = 0; k < nseg; k++) {
    const BatchItem* it = items + segs[k].first;
    const int cnt = std::min(ctas, segs[k].count), ni = segs[k].count;
    if (ni <= 0) continue;
#define GSE_BAS(WW)                                                                          \
  case WW: {                                                                                 \
    static std::atomic<bool> done[64];                                                               \
    const size_t smem = sizeof(int) * ScatterGeom<WW>::words;                                \
    e = set_smem_once(k_batch_adj_scatter<WW>, smem, done);                                  \
    if (e == cudaSuccess)                                                                    \
      k_batch_adj_scatter<WW><<<cnt, kScatterThreads, smem, st>>>(sorted, perm, start, sys,  \
                                                                  it, ni, c, gfx, gfy, gfz,  \
                                                                  grid64);                   \
    break;                                                                                   \
  }
    switch (segs[k].W) {
      GSE_BAS(9)
      GSE_BAS(11)
      GSE_BAS(13)
      GSE_BAS(15)
      default: e = cudaErrorInvalidValue;
    }
#undef GSE_BAS
    if (e != cudaSuccess) return e;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return launch_grid64_to_real(grid64, gsize, lambda, st);
}

cudaError_t launch_batch_adj_gather_tiled(const float4* sorted, const int* perm, const int* start,
                                          const BatchSys* sys, const BatchItem* items,
                                          const BatchSeg* segs, int nseg, int ctas, double c,
                                          const double* dLdE, const float* psi, const float* phi,
                                          const double* gfx, const double* gfy, const double* gfz,
                                          double* dq, double* dx, double* dy, double* dz,
                                          cudaStream_t st) {
  for (int k = 0; k < nseg; k++) {
    const BatchItem* it = items + segs[k].first;
    const int cnt = std::min(ctas, segs[k].count), ni = segs[k].count;
    if (ni <= 0) continue;
    cudaError_t e;
#define GSE_BAG(WW)                                                                          \
  case WW: {                                                                                 \
    static std::atomic<bool> done[64];                                                               \
    const size_t smem = AdjGatherGeom<WW>::bytes;                                            \
    e = set_smem_once(k_batch_adj_gather_tiled<WW>, smem, done);                             \
    if (e == cudaSuccess)                                                                    \
      k_batch_adj_gather_tiled<WW><<<cnt, kAdjThreads, smem, st>>>(                          \
          sorted, perm, start, sys, it, ni, c, dLdE, psi, phi, gfx, gfy, gfz, dq, dx, dy, dz);   \
    break;                                                                                   \
  }
    switch (segs[k].W) {
      GSE_BAG(9)
      GSE_BAG(11)
      GSE_BAG(13)
      GSE_BAG(15)
      default: e = cudaErrorInvalidValue;
    }
#undef GSE_BAG
    if (e != cudaSuccess) return e;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}


// ---------------------------------------------------------------------------
// Reverse pass of a batch in one persistent cooperative launch (grids of at
// most 64 points, multiples of 8, per side): the adjoint source of every
// system into the int64 grid, its solve with the Green's function, and the
// reverse-pass gather.  Reads the forward pass's sorted atoms, bins and
// potential.
// ---------------------------------------------------------------------------
constexpr int kFusedRevThreads = 512;
static_assert(kFusedRevThreads == kScatterThreads, "the fused kernel runs the scatter bricks");

constexpr size_t cmax_rev(size_t a, size_t b) { return a > b ? a : b; }
constexpr size_t fused_rev_smem() {
  return cmax_rev(
      cmax_rev(cmax_rev(sizeof(int) * ScatterGeom<9>::words, sizeof(int) * ScatterGeom<11>::words),
               cmax_rev(sizeof(int) * ScatterGeom<13>::words, sizeof(int) * ScatterGeom<15>::words)),
      cmax_rev(cmax_rev(cmax_rev(AdjGatherGeom<9, kFusedRevThreads>::bytes,
                                 AdjGatherGeom<11, kFusedRevThreads>::bytes),
                        cmax_rev(AdjGatherGeom<13, kFusedRevThreads>::bytes,
                                 AdjGatherGeom<15, kFusedRevThreads>::bytes)),
               sizeof(SmallFftTw) + sizeof(int) * 3 * (kSfSmemSystems + 1)));
}

__global__ void __launch_bounds__(kFusedRevThreads, 1) k_batch_reverse_fused(BatchFused a) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) unsigned char fsm[];
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long gstride = (long long)gridDim.x * blockDim.x;
  for (long long i = gtid; i < a.gtot; i += gstride) a.g64[i] = 0;
  if (gtid < 2) a.qctr[2 + gtid] = 0;
  cg::this_grid().sync();
  for (int it = fused_next_item(&a.qctr[2]); it < a.nscat; it = fused_next_item(&a.qctr[2])) {
    const BatchItem item = a.scat[it];
    const BatchSys& S = a.sys[item.sys];
    const int* st = a.w.start + S.bin_off;
    long long* g = a.g64 + S.grid_off;
    int* tile = reinterpret_cast<int*>(fsm);
    const float cA = (float)(a.ccelec * (double)S.sg.pref);
    switch (S.W) {
      case 9: adj_scatter_brick<9>(a.sorted, a.perm, st, S.b, S.sg, cA, a.gfx, a.gfy, a.gfz,
                                   item.bx, item.by, item.bz, tile, g); break;
      case 11: adj_scatter_brick<11>(a.sorted, a.perm, st, S.b, S.sg, cA, a.gfx, a.gfy, a.gfz,
                                     item.bx, item.by, item.bz, tile, g); break;
      case 13: adj_scatter_brick<13>(a.sorted, a.perm, st, S.b, S.sg, cA, a.gfx, a.gfy, a.gfz,
                                     item.bx, item.by, item.bz, tile, g); break;
      default: adj_scatter_brick<15>(a.sorted, a.perm, st, S.b, S.sg, cA, a.gfx, a.gfy, a.gfz,
                                     item.bx, item.by, item.bz, tile, g); break;
    }
    __syncthreads();
  }
  cg::this_grid().sync();
  fused_solve(a, a.psi, false, fsm);
  cg::this_grid().sync();
  for (int it = fused_next_item(&a.qctr[3]); it < a.nagath; it = fused_next_item(&a.qctr[3])) {
    const BatchItem item = a.agath[it];
    const BatchSys& S = a.sys[item.sys];
    const int* st = a.w.start + S.bin_off;
    const double gE_ch3 = a.dLdE[item.sys] * a.ccelec * S.h3;
    const float* ps = a.psi + S.grid_off;
    const float* ph = a.phi + S.grid_off;
    switch (S.W) {
#define GSE_FAG(WW)                                                                          \
  case WW:                                                                                   \
    adj_gather_brick<WW, kFusedRevThreads>(a.sorted, a.perm, st, S.b, S.sp, S.sg, a.ccelec,  \
                                           gE_ch3, ps, ph, a.gfx, a.gfy, a.gfz, a.dq, a.dx,  \
                                           a.dy, a.dz, item.bx, item.by, item.bz, fsm);      \
    break;
      GSE_FAG(9)
      GSE_FAG(11)
      GSE_FAG(13)
      default:
        adj_gather_brick<15, kFusedRevThreads>(a.sorted, a.perm, st, S.b, S.sp, S.sg, a.ccelec,
                                               gE_ch3, ps, ph, a.gfx, a.gfy, a.gfz, a.dq, a.dx,
                                               a.dy, a.dz, item.bx, item.by, item.bz, fsm);
        break;
#undef GSE_FAG
    }
    __syncthreads();
  }
}

int batch_fused_rev_ctas() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return 0;
  }
  int v = cache[dev].load();
  if (v == 0) {
    const size_t smem = fused_rev_smem();
    int nb = 0;
    if (cudaFuncSetAttribute(k_batch_reverse_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_batch_reverse_fused,
                                                      kFusedRevThreads, smem) != cudaSuccess) {
      cudaGetLastError();
      nb = 0;
    }
    v = nb > 0 ? nb * sm_count() : -1;
    cache[dev].store(v);
  }
  return v > 0 ? v : 0;
}

cudaError_t launch_batch_reverse_fused(const BatchFused& a, int ctas, cudaStream_t st) {
  const int most = batch_fused_rev_ctas();
  if (most <= 0 || ctas < 1 || ctas > most) return cudaErrorCooperativeLaunchTooLarge;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(kFusedRevThreads);
  cfg.dynamicSmemBytes = fused_rev_smem();
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_batch_reverse_fused, a);
}

cudaError_t launch_batch_adj_source(const float4* xyzq, const int* perm, int ntot,
                                    const BatchSys* sys, const int* first, int nsys, double c,
                                    const double* gfx, const double* gfy, const double* gfz,
                                    float* lambda, cudaStream_t st) {
  if (ntot <= 0) return cudaSuccess;
  k_batch_adj_source<<<sm_count() * 16, 256, 0, st>>>(xyzq, perm, ntot, sys, first, nsys, c, gfx, gfy,
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
  k_batch_adj_gather<<<sm_count() * 16, 256, 0, st>>>(xyzq, perm, ntot, sys, first, nsys, c, dLdE, psi,
                                               phi, gfx, gfy, gfz, dq, dx, dy, dz);
  return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_adj_source(const typename Vec4<CT>::type* xyzq, const int* perm, int n,
                              const Stencil<CT>& s, double c, const double* gfx,
                              const double* gfy, const double* gfz, CT* lambda, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int blocks = (int)std::min<long long>(sm_count() * 16, (n + 7) / 8);
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
  const int blocks = (int)std::min<long long>(sm_count() * 16, (n + 7) / 8);
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
