// gse_smallfft.cuh -- 3-D real FFT solve of small periodic grids (every side a
// multiple of 8, at most 64 points) inside a persistent kernel, for the
// batched systems.
//
// A 1-D complex transform of length M = 8 m is done by a group of 8 lanes,
// each holding m values in registers.  With the input index j = m j2 + j1
// (j2 = the lane, j1 = the register) and the output index k = k1 + 8 k2:
//   stage 1: for each j1 an 8-point DFT over j2 across the group's lanes
//            (radix-2 decimation in frequency by shuffles; lane l ends with
//            k1 = bitrev3(l)), then the twiddle w^(j1 k1);
//   stage 2: in each lane, the m-point DFT over j1 giving k2 = 0..m-1.
// w = exp(-2 pi i / M) forward and its conjugate inverse, unnormalised (the
// convention of the reference's FFTW transforms, CpuFFTSolver.cpp:41-64, whose
// c2r normalisation the Green's table carries).  r2c is the complex transform
// of the real row keeping outputs 0..M/2; c2r completes the half spectrum by
// conjugate symmetry and ignores the imaginary parts of the zero and Nyquist
// bins, as FFTW's c2r does.
//
// The solve is five passes of independent lines, each line one group's work:
//   x rows     r2c from the int64 spread grid (at 2^40) into the half spectrum
//   y columns  forward
//   z columns  forward, Green's multiply and k-space energy, inverse
//   y columns  inverse
//   x rows     c2r into the real potential
// The energy of each z column is summed in a fixed order within its group and
// the columns of a system in index order, so energies repeat bit for bit.
#pragma once

#include "gse_internal.cuh"

namespace gse {

constexpr int kSfMax = 64;  // largest grid side

// w^t (dir -1 forward, +1 inverse) from the table tw[t] = (cos, sin)(2 pi t / M).
__device__ __forceinline__ float2 sf_w(const float2* tw, int t, float dir) {
  const float2 w = tw[t];
  return make_float2(w.x, dir * w.y);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 cmad(float2 a, float2 b, float2 c) {
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}

__device__ __forceinline__ int bitrev3(int l) { return ((l & 1) << 2) | (l & 2) | ((l >> 2) & 1); }

// Twiddle tables of M = 8, 16, ..., 64 in shared memory: tw[m-1][t].
struct SmallFftTw {
  float2 tw[kSfMax / 8][kSfMax];
};

__device__ __forceinline__ void sf_build_twiddles(SmallFftTw& T) {
  for (int i = threadIdx.x; i < (kSfMax / 8) * kSfMax; i += blockDim.x) {
    const int m = i / kSfMax + 1, t = i % kSfMax;
    double sn, cs;
    sincospi(2.0 * (double)t / (8.0 * m), &sn, &cs);
    T.tw[m - 1][t] = make_float2((float)cs, (float)sn);
  }
}

// In-register DFT of one group of 8 lanes (l = lane & 7): on entry v[j1] =
// x[m l + j1] for j1 < m, on return v[k2] = X[bitrev3(l) + 8 k2] for k2 < m.
// MM >= m is the same in the whole warp (groups of one warp may work on
// different lengths); every lane of the warp must call it.
template <int MM>
__device__ __forceinline__ void sf8_dft_t(float2 (&v)[8], int m, float dir, const SmallFftTw& T) {
  const int l = threadIdx.x & 7;
  const int M = 8 * m;
  const float2* tw = T.tw[m - 1];
#pragma unroll
  for (int h = 4; h >= 1; h >>= 1) {
    const bool upper = (l & h) != 0;
    const float2 w = sf_w(tw, (l & (h - 1)) * (4 / h) * m, dir);  // w_{2h}^(l mod h)
#pragma unroll
    for (int j1 = 0; j1 < MM; j1++) {
      float2 p;
      p.x = __shfl_xor_sync(0xffffffffu, v[j1].x, h);
      p.y = __shfl_xor_sync(0xffffffffu, v[j1].y, h);
      v[j1] = upper ? cmul(make_float2(p.x - v[j1].x, p.y - v[j1].y), w)
                    : make_float2(v[j1].x + p.x, v[j1].y + p.y);
    }
  }
  const int k1 = bitrev3(l);
  float2 t[MM];
  int e1 = 0;  // j1 k1 mod M
#pragma unroll
  for (int j1 = 0; j1 < MM; j1++) {
    t[j1] = j1 < m ? cmul(v[j1], sf_w(tw, e1, dir)) : make_float2(0.f, 0.f);
    e1 += k1;
    if (e1 >= M) e1 -= M;
  }
#pragma unroll
  for (int k2 = 0; k2 < MM; k2++) {
    float2 acc = t[0];
    int e = 0;  // 8 j1 k2 mod M
#pragma unroll
    for (int j1 = 1; j1 < MM; j1++) {
      e += 8 * k2;
      if (e >= M) e -= M;
      if (j1 < m) acc = cmad(t[j1], sf_w(tw, e, dir), acc);
    }
    v[k2] = acc;
  }
}

__device__ __forceinline__ void sf8_dft(float2 (&v)[8], int m, int mmax, float dir,
                                        const SmallFftTw& T) {
  switch (mmax) {
    case 1: sf8_dft_t<1>(v, m, dir, T); break;
    case 2: sf8_dft_t<2>(v, m, dir, T); break;
    case 3: sf8_dft_t<3>(v, m, dir, T); break;
    case 4: sf8_dft_t<4>(v, m, dir, T); break;
    case 5: sf8_dft_t<5>(v, m, dir, T); break;
    case 6: sf8_dft_t<6>(v, m, dir, T); break;
    case 7: sf8_dft_t<7>(v, m, dir, T); break;
    default: sf8_dft_t<8>(v, m, dir, T); break;
  }
}

// Largest m of the warp (groups of 8 lanes may differ).
__device__ __forceinline__ int sf_warp_mmax(int m) {
#pragma unroll
  for (int o = 8; o < 32; o <<= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  return m;
}

}  // namespace gse
