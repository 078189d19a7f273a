// gse_fft.cu -- the mixed form's own 3-D real FFT solve, for cubic grids of
// M = 16 * N2 points per side (N2 = 4 .. 12; 144^3 is N2 = 9):
//
//   k_own_fft_xy_fwd   one CTA per z plane: int64 (or float) plane -> x r2c of
//                      two real rows per half-warp complex transform -> y
//                      transform of each x' column in shared memory -> rho^
//   k_own_fft_z_green  a CTA per 16 (y, x') columns: z transform, Green's
//                      multiply and k-space energy, inverse z transform
//   k_own_fft_xy_inv   one CTA per z plane: inverse y, then the c2r x transform
//                      of two rows per half-warp complex transform -> phi
//
// It replaces, on that path, the int64 -> float conversion pass, the cuFFT
// r2c and c2r plans (three passes each) and the real-space energy pass: the
// grid crosses memory three times in each direction instead of six, and the
// plane passes keep a whole 144 x 73 complex plane in shared memory.
//
// Every 1-D transform of length N = 16 N2 is done by the 16 lanes of a
// half-warp (Cooley-Tukey with N = N2 x 16): lane n1 holds x[n1 + 16 n2] for
// n2 < N2, takes their N2-point DFT in registers, multiplies by w_N^(n1 k2)
// and finishes with a 16-point decimation-in-frequency transform across the
// lanes by shuffles, after which lane l holds X[k2 + N2 brev4(l)].  Twiddles
// come from tables formed in double.  The transforms are unnormalised and use
// FFTW's signs (forward e^{-2 pi i kn/N}), so the Green's table and the energy
// factor are those of the cuFFT path.
#include "gse_fft.cuh"

#include <atomic>
#include <cmath>
#include <cstdint>
#include <type_traits>
#include <vector>

#include "gse_reduce.cuh"

namespace gse {

// w_N2^m of every supported N2, N2 = kFftMinN2 .. kFftMaxN2 one after the
// other: uniform across the lanes, so read from the constant cache
constexpr int twc_offset(int n2) { return (n2 - kFftMinN2) * (n2 + kFftMinN2 - 1) / 2; }
__constant__ float2 c_twn2[twc_offset(kFftMaxN2 + 1)];

namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

__device__ __forceinline__ int brev4(int l) { return (int)(__brev((unsigned)l) >> 28); }

// Twiddles a lane uses, loaded once per kernel: the lane's w_N^(l k2) and
// its three cross-lane stage factors (spans 16, 8, 4).  c points at w_N2^m in
// constant memory.
template <int N2>
struct LaneTw {
  const float2* c;
  float2 wnk[N2];
  float2 ws[3];
  __device__ __forceinline__ void load(const float2* __restrict__ tw, int l) {
    const float2* twnk = tw;            // [16][N2]
    const float2* tw16 = tw + 16 * N2;  // [16]
    c = c_twn2 + twc_offset(N2);
#pragma unroll
    for (int m = 0; m < N2; m++) wnk[m] = twnk[l * N2 + m];
    // span 2h: lanes with (l & h) take w_{2h}^(l mod h) = w_16^((l mod h) 8/h)
    ws[0] = tw16[(l & 7) * 1];
    ws[1] = tw16[(l & 3) * 2];
    ws[2] = tw16[(l & 1) * 4];
  }
};

template <bool INV>
__device__ __forceinline__ float2 cmul_tw(float2 a, float2 w) {
  // a * w (forward) or a * conj(w) (inverse)
  return INV ? make_float2(fmaf(a.x, w.x, a.y * w.y), fmaf(a.y, w.x, -a.x * w.y)) : cmul(a, w);
}

constexpr int smallest_factor(int n) {
  int p = 2;
  while (n % p) p++;
  return p;
}

// In-register DFT of x[0..N) in natural order (N divides N2), by recursive
// decimation in time: N = P Q with P the smallest prime factor; Q-point DFTs
// of the P residue classes, twiddles w_N^(p k), P-point DFTs across them.
// All twiddles are powers of w_N2 from c[].
template <int N2, bool INV, int N>
__device__ __forceinline__ void dft_reg(float2 (&x)[N], const float2* c) {
  if constexpr (N == 1) {
    return;
  } else if constexpr (N == 2) {
    const float2 a = x[0], b = x[1];
    x[0] = make_float2(a.x + b.x, a.y + b.y);
    x[1] = make_float2(a.x - b.x, a.y - b.y);
  } else if constexpr (N == 3) {
    // X0 = x0 + s, X1,2 = x0 - s/2 -/+ i (sqrt(3)/2) d (forward), s = x1 + x2, d = x1 - x2
    constexpr float kS3 = 0.866025403784438646763723170752936183f;
    const float2 s = make_float2(x[1].x + x[2].x, x[1].y + x[2].y);
    const float2 d = make_float2(x[1].x - x[2].x, x[1].y - x[2].y);
    const float2 t = make_float2(fmaf(-0.5f, s.x, x[0].x), fmaf(-0.5f, s.y, x[0].y));
    const float sg = INV ? -kS3 : kS3;
    const float2 u = make_float2(sg * d.y, -sg * d.x);  // -i sg d
    x[0] = make_float2(x[0].x + s.x, x[0].y + s.y);
    x[1] = make_float2(t.x + u.x, t.y + u.y);
    x[2] = make_float2(t.x - u.x, t.y - u.y);
  } else if constexpr (smallest_factor(N) == N) {
    // other primes: direct sum
    float2 y[N];
#pragma unroll
    for (int j = 0; j < N; j++) {
      float re = x[0].x, im = x[0].y;
#pragma unroll
      for (int p = 1; p < N; p++) {
        const float2 w = c[(p * j * (N2 / N)) % N2];
        const float2 t = cmul_tw<INV>(x[p], w);
        re += t.x;
        im += t.y;
      }
      y[j] = make_float2(re, im);
    }
#pragma unroll
    for (int j = 0; j < N; j++) x[j] = y[j];
  } else {
    constexpr int P = smallest_factor(N), Q = N / P;
    float2 a[P][Q];
#pragma unroll
    for (int p = 0; p < P; p++) {
#pragma unroll
      for (int q = 0; q < Q; q++) a[p][q] = x[p + P * q];
      dft_reg<N2, INV, Q>(a[p], c);
#pragma unroll
      for (int k = 1; k < Q; k++)
        if (p > 0) a[p][k] = cmul_tw<INV>(a[p][k], c[(p * k * (N2 / N)) % N2]);
    }
#pragma unroll
    for (int k = 0; k < Q; k++) {
      float2 b[P];
#pragma unroll
      for (int p = 0; p < P; p++) b[p] = a[p][k];
      dft_reg<N2, INV, P>(b, c);
#pragma unroll
      for (int j = 0; j < P; j++) x[k + Q * j] = b[j];
    }
  }
}

// One complex transform of length 16 N2 by a half-warp (mask: its 16 lanes,
// l: the lane within it).  In: v[n2] = x[l + 16 n2].  Out: v[k2] = X[k2 + N2 brev4(l)].
template <int N2, bool INV>
__device__ __forceinline__ void fft16(float2 (&v)[N2], int l, unsigned mask,
                                      const LaneTw<N2>& t) {
  // N2-point DFT of the lane's own values, then the twiddle w_N^(l k2)
  dft_reg<N2, INV, N2>(v, t.c);
#pragma unroll
  for (int k2 = 1; k2 < N2; k2++) v[k2] = cmul_tw<INV>(v[k2], t.wnk[k2]);
  // 16-point decimation in frequency across the lanes: the lower lane of a
  // pair keeps v + p, the upper one (p - v) w; as sg v + p with sg = -1 on
  // upper lanes and w = 1 on lower lanes the code is the same for every lane
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const int h = 8 >> s;
    const bool up = (l & h) != 0;
    const float sg = up ? -1.f : 1.f;
    float2 w = up ? t.ws[s < 3 ? s : 0] : make_float2(1.f, 0.f);
    if (INV) w.y = -w.y;
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) {
      const float px = __shfl_xor_sync(mask, v[k2].x, h);
      const float py = __shfl_xor_sync(mask, v[k2].y, h);
      const float2 d = make_float2(fmaf(sg, v[k2].x, px), fmaf(sg, v[k2].y, py));
      v[k2] = s < 3 ? cmul(d, w) : d;
    }
  }
}

// 32 half-warps per plane CTA (one CTA per SM: M planes)
constexpr int kPlaneThreads = 512;
constexpr int kHalfWarps = kPlaneThreads / 16;
constexpr int kColThreads = 256;
// resident z-pass CTAs per SM that each size fits without spilling
constexpr int z_blocks(int n2) {
  return (n2 == 4 || n2 == 5 || n2 == 8 || n2 == 9) ? 4 : (n2 == 11 || n2 == 12) ? 2 : 3;
}  // 16 half-warps, one per x' column of a tile

template <int N2>
constexpr size_t plane_smem() {
  // the plane [M][M/2+1] complex and one scratch row of M complex per half-warp
  return sizeof(float2) * ((size_t)(16 * N2) * (8 * N2 + 1) + kHalfWarps * (size_t)(16 * N2));
}

// dst[i] = src[i] for i < count by the whole CTA, kBatch loads per thread
// issued before their stores so that they are in flight together.
constexpr int kBatch = 16;
__device__ __forceinline__ void copy_in(float2* __restrict__ dst, const float2* __restrict__ src,
                                        int count) {
  for (int b0 = threadIdx.x; b0 < count; b0 += kPlaneThreads * kBatch) {
    float2 t[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; b++) {
      const int i = b0 + b * kPlaneThreads;
      t[b] = i < count ? src[i] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int b = 0; b < kBatch; b++) {
      const int i = b0 + b * kPlaneThreads;
      if (i < count) dst[i] = t[b];
    }
  }
}

}  // namespace

template <int N2, bool FIXED>
__global__ void __launch_bounds__(kPlaneThreads, 1)
    k_own_fft_xy_fwd(const long long* __restrict__ g64, const float* __restrict__ rho,
                     double unscale, float* __restrict__ rho_out, float2* __restrict__ rhok,
                     const float2* __restrict__ tw) {
  constexpr int M = 16 * N2, X = M / 2 + 1;  // X is odd: column walks are conflict-free
  extern __shared__ float2 fsm[];
  float2* P = fsm;          // [M][X]
  float2* S = fsm + M * X;  // [kHalfWarps][M]
  const int tid = threadIdx.x, hw = tid >> 4, l = tid & 15;
  const unsigned mask = 0xFFFFu << (tid & 16);
  pdl_trigger();
  LaneTw<N2> lt;
  lt.load(tw, l);
  pdl_wait();
  const long long plane = (long long)M * M;
  const long long z0 = (long long)blockIdx.x * plane;
  float2* Z = S + hw * M;
  // x: rows 2p and 2p+1 as the real and imaginary parts of one transform
  for (int pr = hw; pr < M / 2; pr += kHalfWarps) {
    const long long r0 = z0 + (long long)(2 * pr) * M;
    float2 v[N2];
#pragma unroll
    for (int j = 0; j < N2; j++) {
      const int x = l + 16 * j;
      float a, b;
      if (FIXED) {
        a = (float)((double)g64[r0 + x] * unscale);
        b = (float)((double)g64[r0 + M + x] * unscale);
        if (rho_out) {
          rho_out[r0 + x] = a;
          rho_out[r0 + M + x] = b;
        }
      } else {
        a = rho[r0 + x];
        b = rho[r0 + M + x];
      }
      v[j] = make_float2(a, b);
    }
    fft16<N2, false>(v, l, mask, lt);
    const int k1 = brev4(l);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) Z[k2 + N2 * k1] = v[k2];
    __syncwarp(mask);
    // X_a = (Z[k] + conj Z[M-k]) / 2, X_b = (Z[k] - conj Z[M-k]) / 2i
    float2* Pa = P + (2 * pr) * X;
    float2* Pb = Pa + X;
    for (int k = l; k < X; k += 16) {
      const float2 zk = Z[k], zm = Z[k == 0 ? 0 : M - k];
      Pa[k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      Pb[k] = make_float2(0.5f * (zk.y + zm.y), 0.5f * (zm.x - zk.x));
    }
    __syncwarp(mask);
  }
  __syncthreads();
  // y: each x' column in place
  for (int col = hw; col < X; col += kHalfWarps) {
    float2 v[N2];
#pragma unroll
    for (int j = 0; j < N2; j++) v[j] = P[(l + 16 * j) * X + col];
    fft16<N2, false>(v, l, mask, lt);
    const int k1 = brev4(l);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) P[(k2 + N2 * k1) * X + col] = v[k2];
  }
  __syncthreads();
  float2* out = rhok + (long long)blockIdx.x * M * X;
  for (int i = tid; i < M * X; i += kPlaneThreads) out[i] = P[i];
}

template <int N2>
__global__ void __launch_bounds__(kColThreads, z_blocks(N2))
    k_own_fft_z_green(float2* __restrict__ rhok, const float* __restrict__ tab,
                      const float2* __restrict__ tw, double* __restrict__ partials,
                      unsigned* __restrict__ done, double factor, double* __restrict__ out) {
  constexpr int M = 16 * N2, X = M / 2 + 1;
  __shared__ float2 Q[M][17];
  __shared__ float G[M][17];
  const int tid = threadIdx.x, hw = tid >> 4, l = tid & 15;
  const unsigned mask = 0xFFFFu << (tid & 16);
  pdl_trigger();
  LaneTw<N2> lt;
  lt.load(tw, l);
  pdl_wait();
  // 16 consecutive (y, x') columns, y X + x' in the flattened plane, which is
  // contiguous in every z plane: full tiles across row ends (M X / 16 CTAs)
  const int c0 = blockIdx.x * 16, nx = min(16, M * X - c0);
  const long long zs = (long long)M * X;
  const long long base = c0;
  // M * 16 / kColThreads = N2 elements per thread, all loads issued first
  {
    float2 q[N2];
    float gq[N2];
#pragma unroll
    for (int b = 0; b < N2; b++) {
      const int i = tid + b * kColThreads, zz = i >> 4, xi = i & 15;
      if (xi < nx) {
        q[b] = rhok[zz * zs + base + xi];
        gq[b] = tab[zz * zs + base + xi];
      }
    }
#pragma unroll
    for (int b = 0; b < N2; b++) {
      const int i = tid + b * kColThreads, zz = i >> 4, xi = i & 15;
      if (xi < nx) {
        Q[zz][xi] = q[b];
        G[zz][xi] = gq[b];
      }
    }
  }
  __syncthreads();
  double e = 0.0;
  if (hw < nx) {
    float2 v[N2];
#pragma unroll
    for (int j = 0; j < N2; j++) v[j] = Q[l + 16 * j][hw];
    fft16<N2, false>(v, l, mask, lt);
    const int k1 = brev4(l);
    const int xg = (c0 + hw) % X;
    const double wgt = (xg == 0 || 2 * xg == M) ? 1.0 : 2.0;
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) {
      const int kz = k2 + N2 * k1;
      const float f = G[kz][hw];
      const double re = (double)v[k2].x, im = (double)v[k2].y;
      e += wgt * (double)f * (re * re + im * im);
      Q[kz][hw] = make_float2(v[k2].x * f, v[k2].y * f);
    }
    __syncwarp(mask);
#pragma unroll
    for (int j = 0; j < N2; j++) v[j] = Q[l + 16 * j][hw];
    __syncwarp(mask);
    fft16<N2, true>(v, l, mask, lt);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) Q[k2 + N2 * k1][hw] = v[k2];
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < N2; b++) {
    const int i = tid + b * kColThreads, zz = i >> 4, xi = i & 15;
    if (xi < nx) rhok[zz * zs + base + xi] = Q[zz][xi];
  }
  block_sum_to(e, partials);
  last_block_sum_counter(partials, done, factor, out);
}

template <int N2>
__global__ void __launch_bounds__(kPlaneThreads, 1)
    k_own_fft_xy_inv(const float2* __restrict__ rhok, float* __restrict__ phi,
                     const float2* __restrict__ tw) {
  constexpr int M = 16 * N2, X = M / 2 + 1;
  extern __shared__ float2 fsm[];
  float2* P = fsm;                                     // [M][X]
  float* S = reinterpret_cast<float*>(fsm + M * X);    // [kHalfWarps][2M]
  const int tid = threadIdx.x, hw = tid >> 4, l = tid & 15;
  const unsigned mask = 0xFFFFu << (tid & 16);
  pdl_trigger();
  LaneTw<N2> lt;
  lt.load(tw, l);
  pdl_wait();
  copy_in(P, rhok + (long long)blockIdx.x * M * X, M * X);
  __syncthreads();
  // inverse y: each x' column in place
  for (int col = hw; col < X; col += kHalfWarps) {
    float2 v[N2];
#pragma unroll
    for (int j = 0; j < N2; j++) v[j] = P[(l + 16 * j) * X + col];
    fft16<N2, true>(v, l, mask, lt);
    const int k1 = brev4(l);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) P[(k2 + N2 * k1) * X + col] = v[k2];
  }
  __syncthreads();
  // c2r x: the half spectra A (row 2p) and B (row 2p+1), extended by
  // Hermitian symmetry, combined as A + iB; one inverse transform gives row
  // 2p in the real and row 2p+1 in the imaginary part
  float* T = S + hw * 2 * M;
  float* out = phi + (long long)blockIdx.x * M * M;
  for (int pr = hw; pr < M / 2; pr += kHalfWarps) {
    const float2* Pa = P + (2 * pr) * X;
    const float2* Pb = Pa + X;
    float2 v[N2];
#pragma unroll
    for (int j = 0; j < N2; j++) {
      const int k = l + 16 * j;
      float2 A, B;
      if (2 * k <= M) {
        A = Pa[k];
        B = Pb[k];
        if (k == 0 || 2 * k == M) {
          A.y = 0.f;
          B.y = 0.f;
        }
      } else {
        A = Pa[M - k];
        B = Pb[M - k];
        A.y = -A.y;
        B.y = -B.y;
      }
      v[j] = make_float2(A.x - B.y, A.y + B.x);
    }
    fft16<N2, true>(v, l, mask, lt);
    const int k1 = brev4(l);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) {
      T[k2 + N2 * k1] = v[k2].x;
      T[M + k2 + N2 * k1] = v[k2].y;
    }
    __syncwarp(mask);
    float* ra = out + (long long)(2 * pr) * M;
    for (int i = l; i < M; i += 16) {
      ra[i] = T[i];
      ra[M + i] = T[M + i];
    }
    __syncwarp(mask);
  }
}

// ---------------------------------------------------------------------------
// Plane passes with the plane staged by bulk copies
// ---------------------------------------------------------------------------
// The same transforms, the plane brought into shared memory by the copy
// engine (cp.async.bulk, completion counted on an mbarrier) instead of by
// each lane's loads: the forward pass stages its input in one copy per round
// of x transforms (2 kHalfWarps rows), so a round starts as soon as its rows
// have arrived, and writes the half spectrum over rows it has consumed; the
// inverse pass stages the whole half spectrum in one copy.  Used where the
// plane and the scratch rows fit in shared memory (M <= 144 from the int64
// grid).  Every wait is bounded: past `wait_cycles` (kStageWaitCycles, about a
// second) the CTA sets kFlagStall in `flags` and returns without writing.  A
// test makes the forward pass's first wait run out by expecting `extra_tx`
// bytes more than its copies bring (every copy still completes).
constexpr long long kStageWaitCycles = 2000000000LL;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void stage_bulk(void* dst, const void* src, unsigned bytes,
                                           unsigned long long* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Wait for phase 0 of `bar`; false when `limit` clock cycles pass first.
__device__ __forceinline__ bool stage_wait(unsigned long long* bar, long long limit) {
  const long long t0 = clock64();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_u32(bar))
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}

// Byte layout of the forward pass's shared memory for input element In:
// region A holds the staged input plane at offset `in_off` and, as the
// rounds consume it, the half spectrum P [M][X] from offset 0 (P's rows of
// a round end before the input rows of the next round start); then the
// scratch rows [kHalfWarps][M] complex.
template <int N2, typename In>
struct StagedFwd {
  static constexpr int M = 16 * N2, X = M / 2 + 1;
  static constexpr int kRows = 2 * kHalfWarps;  // rows per round
  static constexpr int kRounds = (M + kRows - 1) / kRows;
  static constexpr long long p_pair = 2LL * X * sizeof(float2), in_pair = 2LL * M * sizeof(In);
  static constexpr long long lag = p_pair > in_pair ? (p_pair - in_pair) * kHalfWarps : 0;
  static constexpr size_t in_off = (size_t)(lag * (kRounds - 1) + 15) / 16 * 16;
  static constexpr size_t in_bytes = sizeof(In) * (size_t)M * M;
  static constexpr size_t p_bytes = sizeof(float2) * (size_t)M * X;
  static constexpr size_t a_bytes =
      ((in_off + in_bytes > p_bytes ? in_off + in_bytes : p_bytes) + 15) / 16 * 16;
  static constexpr size_t bytes = a_bytes + sizeof(float2) * kHalfWarps * (size_t)M;
  static_assert(kRounds <= 3, "three staging barriers");
};

template <int N2, bool FIXED>
__global__ void __launch_bounds__(kPlaneThreads, 1)
    k_own_fft_xy_fwd_staged(const long long* __restrict__ g64, const float* __restrict__ rho,
                            double unscale, float* __restrict__ rho_out,
                            float2* __restrict__ rhok, const float2* __restrict__ tw,
                            int* __restrict__ flags, unsigned extra_tx, long long wait_cycles) {
  typedef typename std::conditional<FIXED, long long, float>::type In;
  typedef StagedFwd<N2, In> L;
  constexpr int M = L::M, X = L::X;
  extern __shared__ __align__(16) unsigned char smb[];
  __shared__ unsigned long long bars[3];
  float2* P = reinterpret_cast<float2*>(smb);                           // [M][X]
  const In* stg = reinterpret_cast<const In*>(smb + L::in_off);        // [M][M]
  float2* S = reinterpret_cast<float2*>(smb + L::a_bytes);              // [kHalfWarps][M]
  const int tid = threadIdx.x, hw = tid >> 4, l = tid & 15;
  const unsigned mask = 0xFFFFu << (tid & 16);
  const long long plane = (long long)M * M;
  const In* src = (FIXED ? reinterpret_cast<const In*>(g64) : reinterpret_cast<const In*>(rho)) +
                  (long long)blockIdx.x * plane;
  pdl_trigger();
  if (tid == 0) {
#pragma unroll
    for (int r = 0; r < L::kRounds; r++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[r])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  LaneTw<N2> lt;
  lt.load(tw, l);
  pdl_wait();
  if (tid == 0) {
#pragma unroll
    for (int r = 0; r < L::kRounds; r++) {
      const int r0 = r * L::kRows, nr = min(L::kRows, M - r0);
      if (r == 0 && extra_tx)
        asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bars[0])),
                     "r"(extra_tx)
                     : "memory");
      stage_bulk(smb + L::in_off + sizeof(In) * (size_t)r0 * M, src + (long long)r0 * M,
                 (unsigned)(sizeof(In) * nr * M), &bars[r]);
    }
  }
  __syncthreads();  // barriers initialised before anyone waits on them
  float2* Z = S + hw * M;
  const long long z0 = (long long)blockIdx.x * plane;
#pragma unroll 1
  for (int r = 0; r < L::kRounds; r++) {
    const bool ok = __syncthreads_and(stage_wait(&bars[r], wait_cycles));
    if (!ok) {
      if (tid == 0 && flags) *flags = kFlagStall;
      return;
    }
    const int pr = r * kHalfWarps + hw;
    const bool has = pr < M / 2;
    float2 v[N2];
    if (has) {
      const In* ra = stg + (2 * pr) * M;
#pragma unroll
      for (int j = 0; j < N2; j++) {
        const int x = l + 16 * j;
        float a, b;
        if (FIXED) {
          a = (float)((double)ra[x] * unscale);
          b = (float)((double)ra[M + x] * unscale);
          if (rho_out) {
            rho_out[z0 + (2 * pr) * M + x] = a;
            rho_out[z0 + (2 * pr + 1) * M + x] = b;
          }
        } else {
          a = ra[x];
          b = ra[M + x];
        }
        v[j] = make_float2(a, b);
      }
    }
    __syncthreads();  // the round's rows are read before P is written over them
    if (has) {
      fft16<N2, false>(v, l, mask, lt);
      const int k1 = brev4(l);
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) Z[k2 + N2 * k1] = v[k2];
      __syncwarp(mask);
      float2* Pa = P + (2 * pr) * X;
      float2* Pb = Pa + X;
      for (int k = l; k < X; k += 16) {
        const float2 zk = Z[k], zm = Z[k == 0 ? 0 : M - k];
        Pa[k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        Pb[k] = make_float2(0.5f * (zk.y + zm.y), 0.5f * (zm.x - zk.x));
      }
      __syncwarp(mask);
    }
  }
  __syncthreads();
  for (int col = hw; col < X; col += kHalfWarps) {
    float2 v[N2];
#pragma unroll
    for (int j = 0; j < N2; j++) v[j] = P[(l + 16 * j) * X + col];
    fft16<N2, false>(v, l, mask, lt);
    const int k1 = brev4(l);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) P[(k2 + N2 * k1) * X + col] = v[k2];
  }
  __syncthreads();
  float2* out = rhok + (long long)blockIdx.x * M * X;
  for (int i = tid; i < M * X; i += kPlaneThreads) out[i] = P[i];
}

template <int N2>
__global__ void __launch_bounds__(kPlaneThreads, 1)
    k_own_fft_xy_inv_staged(const float2* __restrict__ rhok, float* __restrict__ phi,
                            const float2* __restrict__ tw, int* __restrict__ flags) {
  constexpr int M = 16 * N2, X = M / 2 + 1;
  extern __shared__ __align__(16) unsigned char smb[];
  __shared__ unsigned long long bar;
  float2* P = reinterpret_cast<float2*>(smb);                                  // [M][X]
  float* S = reinterpret_cast<float*>(smb + sizeof(float2) * (size_t)M * X);   // [kHalfWarps][2M]
  const int tid = threadIdx.x, hw = tid >> 4, l = tid & 15;
  const unsigned mask = 0xFFFFu << (tid & 16);
  pdl_trigger();
  LaneTw<N2> lt;
  lt.load(tw, l);
  pdl_wait();
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    stage_bulk(P, rhok + (long long)blockIdx.x * M * X, (unsigned)(sizeof(float2) * M * X), &bar);
  }
  __syncthreads();
  if (!__syncthreads_and(stage_wait(&bar, kStageWaitCycles))) {
    if (tid == 0 && flags) *flags = kFlagStall;
    return;
  }
  for (int col = hw; col < X; col += kHalfWarps) {
    float2 v[N2];
#pragma unroll
    for (int j = 0; j < N2; j++) v[j] = P[(l + 16 * j) * X + col];
    fft16<N2, true>(v, l, mask, lt);
    const int k1 = brev4(l);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) P[(k2 + N2 * k1) * X + col] = v[k2];
  }
  __syncthreads();
  float* T = S + hw * 2 * M;
  float* out = phi + (long long)blockIdx.x * M * M;
  for (int pr = hw; pr < M / 2; pr += kHalfWarps) {
    const float2* Pa = P + (2 * pr) * X;
    const float2* Pb = Pa + X;
    float2 v[N2];
#pragma unroll
    for (int j = 0; j < N2; j++) {
      const int k = l + 16 * j;
      float2 A, B;
      if (2 * k <= M) {
        A = Pa[k];
        B = Pb[k];
        if (k == 0 || 2 * k == M) {
          A.y = 0.f;
          B.y = 0.f;
        }
      } else {
        A = Pa[M - k];
        B = Pb[M - k];
        A.y = -A.y;
        B.y = -B.y;
      }
      v[j] = make_float2(A.x - B.y, A.y + B.x);
    }
    fft16<N2, true>(v, l, mask, lt);
    const int k1 = brev4(l);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) {
      T[k2 + N2 * k1] = v[k2].x;
      T[M + k2 + N2 * k1] = v[k2].y;
    }
    __syncwarp(mask);
    float* ra = out + (long long)(2 * pr) * M;
    for (int i = l; i < M; i += 16) {
      ra[i] = T[i];
      ra[M + i] = T[M + i];
    }
    __syncwarp(mask);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
bool own_fft_supported(const int M[3]) {
  if (M[0] != M[1] || M[0] != M[2] || M[0] % 16 != 0) return false;
  const int n2 = M[0] / 16;
  return n2 >= kFftMinN2 && n2 <= kFftMaxN2;
}

cudaError_t make_fft_twiddles(int M, float2** out) {
  const int n2 = M / 16;
  if (n2 < kFftMinN2 || n2 > kFftMaxN2 || M % 16) return cudaErrorInvalidValue;
  std::vector<float2> h(16 * n2 + 16 + n2);
  auto w = [](long long m, int n) {
    const double a = -2.0 * kPi * (double)(m % n) / (double)n;
    return make_float2((float)std::cos(a), (float)std::sin(a));
  };
  for (int n1 = 0; n1 < 16; n1++)
    for (int k2 = 0; k2 < n2; k2++) h[n1 * n2 + k2] = w((long long)n1 * k2, M);
  for (int m = 0; m < 16; m++) h[16 * n2 + m] = w(m, 16);
  for (int m = 0; m < n2; m++) h[16 * n2 + 16 + m] = w(m, n2);
  // this size's w_N2^m into the constant table (of the current device)
  cudaError_t e = cudaMemcpyToSymbol(c_twn2, h.data() + 16 * n2 + 16, sizeof(float2) * n2,
                                     sizeof(float2) * twc_offset(n2));
  if (e != cudaSuccess) return e;
  e = cudaMalloc(out, sizeof(float2) * h.size());
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*out, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice);
}

namespace {

// Opt each plane kernel in to its shared memory once per device.
template <typename K>
cudaError_t allow_smem(K kernel, size_t bytes, std::atomic<bool> (&done)[64]) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!done[dev]) {
    const cudaError_t e =
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    done[dev] = true;
  }
  return cudaSuccess;
}

// Largest dynamic shared memory a block may opt in to on the current device.
size_t optin_smem() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  int v = cache[dev].load();
  if (v == 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
      return 0;
    cache[dev] = v;
  }
  return (size_t)v;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

template <int N2>
cudaError_t fwd_n2(const long long* g64, const float* rho, double unscale, float* rho_out,
                   float2* rhok, const float2* tw, int* flags, bool pdl, bool stall_test,
                   cudaStream_t st) {
  const unsigned extra = stall_test ? 16u : 0u;
  const long long cycles = stall_test ? 2000000LL : kStageWaitCycles;
  constexpr int M = 16 * N2;
  constexpr size_t smem = plane_smem<N2>();
  static std::atomic<bool> fx[64], fl[64], sx[64], sl[64];
  if (aligned16(g64 ? (const void*)g64 : (const void*)rho)) {
    if (g64 && StagedFwd<N2, long long>::bytes <= optin_smem()) {
      constexpr size_t sm = StagedFwd<N2, long long>::bytes;
      cudaError_t e = allow_smem(k_own_fft_xy_fwd_staged<N2, true>, sm, sx);
      if (e != cudaSuccess) return e;
      e = launch_dependent(pdl, k_own_fft_xy_fwd_staged<N2, true>, dim3(M), dim3(kPlaneThreads),
                           sm, st, g64, rho, unscale, rho_out, rhok, tw, flags, extra, cycles);
      return e != cudaSuccess ? e : cudaGetLastError();
    }
    if (!g64 && StagedFwd<N2, float>::bytes <= optin_smem()) {
      constexpr size_t sm = StagedFwd<N2, float>::bytes;
      cudaError_t e = allow_smem(k_own_fft_xy_fwd_staged<N2, false>, sm, sl);
      if (e != cudaSuccess) return e;
      e = launch_dependent(pdl, k_own_fft_xy_fwd_staged<N2, false>, dim3(M),
                           dim3(kPlaneThreads), sm, st, g64, rho, unscale, rho_out, rhok, tw,
                           flags, extra, cycles);
      return e != cudaSuccess ? e : cudaGetLastError();
    }
  }
  if (g64) {
    cudaError_t e = allow_smem(k_own_fft_xy_fwd<N2, true>, smem, fx);
    if (e != cudaSuccess) return e;
    e = launch_dependent(pdl, k_own_fft_xy_fwd<N2, true>, dim3(M), dim3(kPlaneThreads), smem,
                         st, g64, rho, unscale, rho_out, rhok, tw);
    if (e != cudaSuccess) return e;
  } else {
    cudaError_t e = allow_smem(k_own_fft_xy_fwd<N2, false>, smem, fl);
    if (e != cudaSuccess) return e;
    e = launch_dependent(pdl, k_own_fft_xy_fwd<N2, false>, dim3(M), dim3(kPlaneThreads), smem,
                         st, g64, rho, unscale, rho_out, rhok, tw);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

template <int N2>
cudaError_t z_n2(float2* rhok, const float* tab, const float2* tw, double* partials,
                 unsigned* done, double factor, double* out, bool pdl, cudaStream_t st) {
  constexpr int M = 16 * N2, X = M / 2 + 1;
  const cudaError_t e = launch_dependent(pdl, k_own_fft_z_green<N2>, dim3((M * X + 15) / 16),
                                         dim3(kColThreads), 0, st, rhok, tab, tw, partials, done,
                                         factor, out);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <int N2>
cudaError_t inv_n2(const float2* rhok, float* phi, const float2* tw, int* flags, bool pdl,
                   cudaStream_t st) {
  constexpr int M = 16 * N2;
  constexpr size_t smem = plane_smem<N2>();
  static std::atomic<bool> fi[64], si[64];
  if (aligned16(rhok) && smem <= optin_smem()) {
    cudaError_t e = allow_smem(k_own_fft_xy_inv_staged<N2>, smem, si);
    if (e != cudaSuccess) return e;
    e = launch_dependent(pdl, k_own_fft_xy_inv_staged<N2>, dim3(M), dim3(kPlaneThreads), smem,
                         st, rhok, phi, tw, flags);
    return e != cudaSuccess ? e : cudaGetLastError();
  }
  cudaError_t e = allow_smem(k_own_fft_xy_inv<N2>, smem, fi);
  if (e != cudaSuccess) return e;
  e = launch_dependent(pdl, k_own_fft_xy_inv<N2>, dim3(M), dim3(kPlaneThreads), smem, st, rhok,
                       phi, tw);
  return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace

#define GSE_FFT_SWITCH(CALL)                                                                   \
  switch (M / 16) {                                                                            \
    case 4: return CALL(4);                                                                    \
    case 5: return CALL(5);                                                                    \
    case 6: return CALL(6);                                                                    \
    case 7: return CALL(7);                                                                    \
    case 8: return CALL(8);                                                                    \
    case 9: return CALL(9);                                                                    \
    case 10: return CALL(10);                                                                  \
    case 11: return CALL(11);                                                                  \
    case 12: return CALL(12);                                                                  \
  }                                                                                            \
  return cudaErrorInvalidValue;

cudaError_t launch_own_fft_xy_forward(int M, const long long* g64, const float* rho,
                                      double unscale, float* rho_out, float2* rhok,
                                      const float2* tw, int* flags, bool pdl, bool stall_test,
                                      cudaStream_t st) {
  if (M % 16) return cudaErrorInvalidValue;
#define CALL_FWD(N) fwd_n2<N>(g64, rho, unscale, rho_out, rhok, tw, flags, pdl, stall_test, st)
  GSE_FFT_SWITCH(CALL_FWD)
#undef CALL_FWD
}

cudaError_t launch_own_fft_z_green(int M, float2* rhok, const float* tab, const float2* tw,
                                   double* partials, unsigned* done, double factor,
                                   double* energy_out, bool pdl, cudaStream_t st) {
  if (M % 16) return cudaErrorInvalidValue;
#define CALL_Z(N) z_n2<N>(rhok, tab, tw, partials, done, factor, energy_out, pdl, st)
  GSE_FFT_SWITCH(CALL_Z)
#undef CALL_Z
}

cudaError_t launch_own_fft_xy_inverse(int M, const float2* rhok, float* phi, const float2* tw,
                                      int* flags, bool pdl, cudaStream_t st) {
  if (M % 16) return cudaErrorInvalidValue;
#define CALL_INV(N) inv_n2<N>(rhok, phi, tw, flags, pdl, st)
  GSE_FFT_SWITCH(CALL_INV)
#undef CALL_INV
}

#undef GSE_FFT_SWITCH

}  // namespace gse
