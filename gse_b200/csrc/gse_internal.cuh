// gse_internal.cuh -- shared types and device helpers of the GSE-k library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cmath>

namespace gse {

// Programmatic dependent launch between consecutive kernels of this library
// on one stream: a kernel launched by launch_dependent() may be scheduled
// while its predecessor is still running; it runs its own set-up, then
// pdl_wait() returns once the predecessor has completed and its writes are
// visible.  Every kernel so launched calls pdl_wait() on every path before
// it reads a predecessor's output or exits, so completion carries down the
// chain.  pdl_trigger() lets the successor be scheduled once every block of
// the current kernel has started.  Both are no-ops for a normal launch.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launch `kernel` on `st` after the kernel before it on the stream, with
// programmatic serialisation when `pdl` (the kernel must call pdl_wait()).
template <typename... KArgs, typename... Args>
cudaError_t launch_dependent(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block,
                             size_t smem, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Streaming multiprocessors of the current device (148 on a B200), looked up
// once per device; grid-stride kernels size their grids as multiples of it.
inline int sm_count() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return 148;
  }
  int v = cache[dev].load(std::memory_order_relaxed);
  if (v <= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
      cudaGetLastError();
      v = 148;
    }
    cache[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

constexpr double kPi = 3.14159265358979323846;  // pi_dbl, TypesGSE.h:24
constexpr int kMaxStencil = 64;                  // max 2n+1 per axis

template <typename CT> struct Vec4;
template <> struct Vec4<double> { typedef double4 type; };
template <> struct Vec4<float> { typedef float4 type; };

template <typename CT> struct Cplx;
template <> struct Cplx<double> { typedef double2 type; };
template <> struct Cplx<float> { typedef float2 type; };

// Stencil constants of one spread or gather call, derived on the host exactly
// as CpuGaussCharge computes them (CpuGaussCharge.cpp:114-128 and :244-258):
// the spacing and its inverse in double, then cast to CT.
// Values of a context's status flag (a host-mapped int that kernels set and the
// host reads after a synchronisation).
constexpr int kFlagNonFinite = 1;  // a position or charge is NaN or infinite
constexpr int kFlagRange = 2;      // a brick's charge overflows the mixed form's tile range
constexpr int kFlagStall = 4;      // a bounded wait in a kernel gave up

template <typename CT>
struct Stencil {
  int M[3];      // grid sizes
  int nst[3];    // n = ceil(rcut / h) per axis
  CT h[3];       // (CT)(box/M)
  CT inv_h[3];   // (CT)(1.0 / (box/M))
  CT rcut2;      // (CT)(rcut*rcut)
  CT inv_2s2;    // (CT)(1/(2 sigma^2))
  CT pref;       // spread: (CT)(2 pi sigma^2)^(-3/2); gather: (CT)((2 pi)^(-3/2) h^3 sigma^-5)
  CT norm_pref1; // (CT)sqrt(2 pi sigma^2), used when normalize != 0
  int normalize;
  double fixed_scale;  // mixed form: fixed-point units per unit charge density
};

template <typename CT>
inline Stencil<CT> make_stencil(const int M[3], const double box[3], double sigma, double rcut,
                                bool gather, bool normalize, double fixed_scale) {
  Stencil<CT> s;
  double hd[3];
  for (int d = 0; d < 3; d++) {
    s.M[d] = M[d];
    hd[d] = box[d] / (double)M[d];
    s.nst[d] = (int)std::ceil(rcut / hd[d]);
    s.h[d] = (CT)hd[d];
    s.inv_h[d] = (CT)(1.0 / hd[d]);
  }
  s.rcut2 = (CT)(rcut * rcut);
  s.inv_2s2 = (CT)(1.0 / (2.0 * sigma * sigma));
  if (gather)
    s.pref = (CT)(std::pow(2.0 * kPi, -3.0 / 2.0) * hd[0] * hd[1] * hd[2] * std::pow(sigma, -5.0));
  else
    s.pref = (CT)std::pow(2.0 * kPi * sigma * sigma, -3.0 / 2.0);
  s.norm_pref1 = (CT)std::sqrt(2.0 * kPi * sigma * sigma);
  s.normalize = normalize ? 1 : 0;
  s.fixed_scale = fixed_scale;
  return s;
}

// Fixed-point units per unit charge density for the mixed form's int64 grid:
// 2^40 for the default widths; coarser when a narrow Gaussian makes single
// contributions large, so that any sum of up to 2^22 maximal contributions
// stays inside int64.
inline double fixed_scale_for(double spread_pref) {
  int k = 40;
  double m = std::fabs(spread_pref) / 0.05;
  while (m > 1.0 && k > 8) {
    m *= 0.5;
    k--;
  }
  return std::ldexp(1.0, k);
}

// ---- round-to-nearest arithmetic that nvcc may not contract into FMAs ----
// The stencil origin and the spherical cut must be bit-identical to the
// reference's separately rounded products and sums.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

// C round(): halfway cases away from zero (the reference calls round()).
__device__ __forceinline__ int round_to_int(double v) { return (int)round(v); }
__device__ __forceinline__ int round_to_int(float v) { return (int)roundf(v); }

__device__ __forceinline__ double gexp(double v) { return exp(v); }
__device__ __forceinline__ float gexp(float v) { return expf(v); }
// Stencil weights of the forward spread and gather: exp in the FP64 form; in
// the mixed form the hardware exponential (__expf: ex2.approx of x log2 e),
// within about 1e-6 relative for the exponents of these stencils (|x| < 40),
// which moves the mixed forces against the FP64 reference by less than 1e-7.
__device__ __forceinline__ double wexp(double v) { return exp(v); }
__device__ __forceinline__ float wexp(float v) { return __expf(v); }

__device__ __forceinline__ int pmod(int a, int m) {
  int r = a % m;
  return r < 0 ? r + m : r;
}

// pmod for values that are almost always within one period of [0, m)
__device__ __forceinline__ int wrap1(int a, int m) {
  if (a >= 0 && a < m) return a;
  if (a < 0 && a >= -m) return a + m;
  if (a >= m && a < 2 * m) return a - m;
  return pmod(a, m);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace gse
