// gse_probe.cu -- measured arithmetic rates of the GPU the library runs on.
//
// The spread and gather kernels are bound by FP32 arithmetic and instruction
// issue, not by HBM bandwidth, so a roofline for them needs the FP32 rate this
// GPU reaches at its current clocks.  gse_measure_fp32_rate times a kernel of
// independent FP32 fused multiply-adds (scalar and packed f32x2 forms, the
// faster one counts) over every SM and reports the rate it sustained.
#include <algorithm>

#include "gse_b200.h"
#include "gse_internal.cuh"

namespace gse {
gse_status_t set_error(gse_status_t s, const char* msg);
}

namespace {

constexpr int kChains = 8;     // independent accumulators per thread
constexpr int kIters = 2048;   // loop trips per launch
constexpr int kThreads = 256;

// kChains * kIters fmas per thread; the result is stored only if it is an
// impossible value, so the compiler keeps the arithmetic and the store stays
// off the memory path.
__global__ void __launch_bounds__(kThreads) k_fma_scalar(float a, float b, float* sink) {
  float acc[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) acc[c] = (float)(threadIdx.x + c);
  for (int i = 0; i < kIters; i++) {
#pragma unroll
    for (int c = 0; c < kChains; c++) acc[c] = fmaf(acc[c], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; c++) s += acc[c];
  if (s == -1.2345e30f) sink[threadIdx.x] = s;
}

// The same with the packed two-lane form (two fmas per instruction).
__global__ void __launch_bounds__(kThreads) k_fma_packed(float a, float b, float* sink) {
  unsigned long long acc[kChains / 2], a2, b2;
  asm("mov.b64 %0, {%1, %1};" : "=l"(a2) : "f"(a));
  asm("mov.b64 %0, {%1, %1};" : "=l"(b2) : "f"(b));
#pragma unroll
  for (int c = 0; c < kChains / 2; c++) {
    const float x = (float)(threadIdx.x + c), y = x + 0.5f;
    asm("mov.b64 %0, {%1, %2};" : "=l"(acc[c]) : "f"(x), "f"(y));
  }
  for (int i = 0; i < kIters; i++) {
#pragma unroll
    for (int c = 0; c < kChains / 2; c++)
      asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(acc[c]) : "l"(a2), "l"(b2));
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains / 2; c++) {
    float x, y;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(acc[c]));
    s += x + y;
  }
  if (s == -1.2345e30f) sink[threadIdx.x] = s;
}

}  // namespace

extern "C" gse_status_t gse_measure_fp32_rate(int device, void* stream, double* tflops,
                                              double* tflops_packed) {
  using namespace gse;
  if (!tflops) return set_error(GSE_ERR_INVALID_ARG, "NULL tflops");
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return set_error(GSE_ERR_UNSUPPORTED, "no such CUDA device");
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int blocks = sm_count() * 8;  // 2048 threads per SM
  const double flops = 2.0 * kChains * (double)kIters * kThreads * blocks;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float* sink = nullptr;
  gse_status_t status = GSE_OK;
  double best[2] = {0.0, 0.0};
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
      cudaMalloc(&sink, sizeof(float) * kThreads) != cudaSuccess) {
    cudaGetLastError();
    status = set_error(GSE_ERR_CUDA, "event or scratch allocation failed");
  }
  for (int form = 0; form < 2 && status == GSE_OK; form++) {
    for (int rep = 0; rep < 6; rep++) {  // the first launches warm the clocks up
      cudaEventRecord(e0, st);
      if (form == 0)
        k_fma_scalar<<<blocks, kThreads, 0, st>>>(1.0000001f, 1e-7f, sink);
      else
        k_fma_packed<<<blocks, kThreads, 0, st>>>(1.0000001f, 1e-7f, sink);
      cudaEventRecord(e1, st);
      float ms = 0.f;
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        cudaGetLastError();
        status = set_error(GSE_ERR_CUDA, "timing the FP32 rate kernel failed");
        break;
      }
      if (ms > 0.f) best[form] = std::max(best[form], flops / (ms * 1e-3) / 1e12);
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (sink) cudaFree(sink);
  if (status != GSE_OK) return status;
  *tflops = best[0];
  if (tflops_packed) *tflops_packed = best[1];
  return GSE_OK;
}
