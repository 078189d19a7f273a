// gse_ewald.cu -- FP64 Ewald reciprocal-space sum on the GPU.
//
// CpuEwaldRecip::calcForceEnergy (CpuEwaldRecip.cpp:87-147):
//   E   = sum_{k != 0, |k|_int^2 <= kcut^2} P(k) |S(k)|^2,
//   P   = (2 pi / V) ccelec exp(-sigma^2 k^2 / 2) / k^2,
//   S   = sum_i q_i exp(i k . r_i),
//   F_i = sum_k 2 P q_i k Im(conj(S) exp(i k . r_i))   (= -dE/dr_i).
// k and -k contribute equally; the sums run over the half space
// (kz > 0, or kz = 0 and ky > 0, or kz = ky = 0 and kx > 0) and are doubled.
// Rows of constant (ky, kz) are the unit of work: along a row the phase
// exp(i kx 2 pi x / Lx) advances by a complex multiply.
#include <cuda_runtime.h>
#include <math.h>

#include <vector>

#include "gse_ewald.cuh"
#include "gse_internal.cuh"

namespace gse {

constexpr int kEwTile = 64;      // atoms per shared-memory tile (4 builder threads each)
constexpr int kEwThreads = 256;  // == 4 * kEwTile
constexpr int kEwKPerThread = 2; // kx values per thread: rows of up to 512 values

struct EwRow {
  int ky, kz, kx0, nk;  // kx = kx0 .. kx0 + nk - 1
  long long off;         // first S(k) slot of the row
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// PS(k) = P(k) S(k) for every k of one row, and the row's share of the
// energy.  Atoms go through shared memory in tiles; four threads per atom
// build its table exp(i m 2 pi x / Lx), m = 0..kmax, by recurrence from four
// directly evaluated starting points.
__global__ void __launch_bounds__(kEwThreads)
    k_ewald_structure(const double4* __restrict__ xyzq, int n, const EwRow* __restrict__ rows,
                      EwGeom g, int kmax, double2* __restrict__ PS,
                      double* __restrict__ row_energy) {
  extern __shared__ double2 ew_sm[];
  double2* T = ew_sm;                        // [kEwTile][kmax + 1]
  double2* R = ew_sm + kEwTile * (kmax + 1);  // [kEwTile]
  const int pitch = kmax + 1;
  const EwRow row = rows[blockIdx.x];
  const int tid = threadIdx.x;
  const int kxm = max(row.kx0 + row.nk - 1, -row.kx0);
  const int seg = (kxm + 1 + 3) / 4;  // table entries per builder thread
  double2 acc[kEwKPerThread];
#pragma unroll
  for (int j = 0; j < kEwKPerThread; j++) acc[j] = make_double2(0.0, 0.0);
  for (int a0 = 0; a0 < n; a0 += kEwTile) {
    {
      const int at = tid >> 2, part = tid & 3;  // 4 builders per atom
      const int a = a0 + at;
      double4 p = make_double4(0.0, 0.0, 0.0, 0.0);
      if (a < n) p = xyzq[a];
      if (part == 0) {
        const double ang = 2.0 * kPi * ((double)row.ky * p.y * g.inv_box[1] +
                                        (double)row.kz * p.z * g.inv_box[2]);
        double sn, cs;
        sincos(ang, &sn, &cs);
        R[at] = make_double2(p.w * cs, p.w * sn);
      }
      const double th = 2.0 * kPi * p.x * g.inv_box[0];
      double su, cu;
      sincos(th, &su, &cu);
      const double2 u = make_double2(cu, su);
      const int m0 = part * seg, m1 = min(kxm + 1, m0 + seg);
      if (m0 < m1) {
        double s0, c0;
        sincos((double)m0 * th, &s0, &c0);
        double2 t = make_double2(c0, s0);
        for (int m = m0; m < m1; m++) {
          T[at * pitch + m] = t;
          t = cmul(t, u);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kEwKPerThread; j++) {
      const int i = tid + j * kEwThreads;
      if (i < row.nk) {
        const int kx = row.kx0 + i;
        const int m = kx < 0 ? -kx : kx;
        const double sg = kx < 0 ? -1.0 : 1.0;
        double2 s = acc[j];
        for (int a = 0; a < kEwTile; a++) {
          const double2 tt = T[a * pitch + m];
          const double2 r = R[a];
          // r * conj^(kx<0)(tt)
          s.x += r.x * tt.x - r.y * (sg * tt.y);
          s.y += r.x * (sg * tt.y) + r.y * tt.x;
        }
        acc[j] = s;
      }
    }
    __syncthreads();
  }
  double e = 0.0;
#pragma unroll
  for (int j = 0; j < kEwKPerThread; j++) {
    const int i = tid + j * kEwThreads;
    if (i < row.nk) {
      const int kx = row.kx0 + i;
      const double kxv = 2.0 * kPi * kx * g.inv_box[0];
      const double kyv = 2.0 * kPi * row.ky * g.inv_box[1];
      const double kzv = 2.0 * kPi * row.kz * g.inv_box[2];
      const double ksq = kxv * kxv + kyv * kyv + kzv * kzv;
      const double P = g.pref * exp(-ksq * g.half_sigmasq) / ksq;
      PS[row.off + i] = make_double2(P * acc[j].x, P * acc[j].y);
      e += 2.0 * P * (acc[j].x * acc[j].x + acc[j].y * acc[j].y);
    }
  }
  __shared__ double red[kEwThreads / 32];
  e = warp_sum(e);
  if ((tid & 31) == 0) red[tid >> 5] = e;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < kEwThreads / 32; w++) t += red[w];
    row_energy[blockIdx.x] = t;
  }
}

// F_i = sum over the half space of 4 q_i k Im(conj(PS(k)) exp(i k . r_i));
// thread per atom.
__global__ void __launch_bounds__(128)
    k_ewald_force(const double4* __restrict__ xyzq, int n, const EwRow* __restrict__ rows,
                  int nrows, EwGeom g, const double2* __restrict__ PS, double* __restrict__ fx,
                  double* __restrict__ fy, double* __restrict__ fz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = xyzq[i];
  double sx, cx;
  sincos(2.0 * kPi * p.x * g.inv_box[0], &sx, &cx);
  const double2 u = make_double2(cx, sx);
  const double kx1 = 2.0 * kPi * g.inv_box[0];
  double fxa = 0.0, fya = 0.0, fza = 0.0;
  for (int r = 0; r < nrows; r++) {
    const EwRow row = rows[r];
    const double ang = 2.0 * kPi * ((double)row.kx0 * p.x * g.inv_box[0] +
                                    (double)row.ky * p.y * g.inv_box[1] +
                                    (double)row.kz * p.z * g.inv_box[2]);
    double sn, cs;
    sincos(ang, &sn, &cs);
    double2 e = make_double2(cs, sn);
    double ax = 0.0, ayz = 0.0;
    const double2* ps = PS + row.off;
    for (int j = 0; j < row.nk; j++) {
      const double2 s = ps[j];
      const double im = s.x * e.y - s.y * e.x;  // Im(conj(PS) e)
      ax += im * (double)(row.kx0 + j);
      ayz += im;
      e = cmul(e, u);
    }
    fxa += ax * kx1;
    fya += ayz * 2.0 * kPi * row.ky * g.inv_box[1];
    fza += ayz * 2.0 * kPi * row.kz * g.inv_box[2];
  }
  fx[i] = 4.0 * p.w * fxa;
  fy[i] = 4.0 * p.w * fya;
  fz[i] = 4.0 * p.w * fza;
}

std::vector<EwRowHost> ewald_rows(int kcut) {
  std::vector<EwRowHost> rows;
  const int kc2 = kcut * kcut;
  long long off = 0;
  for (int kz = 0; kz <= kcut; kz++)
    for (int ky = (kz == 0 ? 0 : -kcut); ky <= kcut; ky++) {
      const int rem = kc2 - ky * ky - kz * kz;
      if (rem < 0) continue;
      int kxm = (int)std::floor(std::sqrt((double)rem));
      while (kxm * kxm > rem) kxm--;
      while ((kxm + 1) * (kxm + 1) <= rem) kxm++;
      const int kx0 = (kz == 0 && ky == 0) ? 1 : -kxm;
      const int nk = kxm - kx0 + 1;
      if (nk <= 0) continue;
      rows.push_back({ky, kz, kx0, nk, off});
      off += nk;
    }
  return rows;
}

cudaError_t launch_ewald(const double4* xyzq, int n, const std::vector<EwRowHost>& rows,
                         const EwGeom& g, EwScratch w, double* fx, double* fy, double* fz,
                         cudaStream_t st) {
  static_assert(sizeof(EwRowHost) == sizeof(EwRow), "row layout");
  const int nrows = (int)rows.size();
  if (nrows == 0) return cudaSuccess;
  cudaError_t e = cudaMemcpyAsync(w.rows, rows.data(), sizeof(EwRow) * nrows,
                                  cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  int kmax = 0;
  for (const EwRowHost& r : rows) kmax = std::max(kmax, std::max(r.kx0 + r.nk - 1, -r.kx0));
  const size_t smem = sizeof(double2) * ((size_t)kEwTile * (kmax + 1) + kEwTile);
  if (smem > 227 * 1024 || 2 * kmax + 1 > kEwThreads * kEwKPerThread) return cudaErrorInvalidValue;
  e = cudaFuncSetAttribute(k_ewald_structure, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
  if (e != cudaSuccess) return e;
  k_ewald_structure<<<nrows, kEwThreads, smem, st>>>(xyzq, n, (const EwRow*)w.rows, g, kmax,
                                                     w.S, w.row_energy);
  if (fx) {
    k_ewald_force<<<(n + 127) / 128, 128, 0, st>>>(xyzq, n, (const EwRow*)w.rows, nrows, g, w.S,
                                                   fx, fy, fz);
  }
  return cudaGetLastError();
}

}  // namespace gse
