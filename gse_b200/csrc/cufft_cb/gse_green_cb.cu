// gse_green_cb.cu -- load callbacks of the c2r transform of the GSE-k solve.
//
// Compiled on its own to LTO intermediate code (nvcc -dc -fatbin with
// code=lto_100a) and handed to cuFFT with cufftXtSetJITCallback, which links
// it into the transform's kernels: the transform reads each half-spectrum
// element of rho(k) already multiplied by the Green's function table G(k)
// (CpuGreensFuncGSE<T>::mul, CpuGreensFuncGSE.cpp:9-57), so the multiply costs
// no pass of its own.  callerInfo is the device table, one entry per element
// of the half spectrum, in the same order.
#include <cufftXt.h>

__device__ cufftComplex gse_green_load_c(void* dataIn, unsigned long long offset,
                                         void* callerInfo, void* sharedPointer) {
  const cufftComplex v = static_cast<const cufftComplex*>(dataIn)[offset];
  const float g = static_cast<const float*>(callerInfo)[offset];
  cufftComplex r;
  r.x = v.x * g;
  r.y = v.y * g;
  return r;
}

__device__ cufftDoubleComplex gse_green_load_z(void* dataIn, unsigned long long offset,
                                               void* callerInfo, void* sharedPointer) {
  const cufftDoubleComplex v = static_cast<const cufftDoubleComplex*>(dataIn)[offset];
  const double g = static_cast<const double*>(callerInfo)[offset];
  cufftDoubleComplex r;
  r.x = v.x * g;
  r.y = v.y * g;
  return r;
}
