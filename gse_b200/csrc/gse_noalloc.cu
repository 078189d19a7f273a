// gse_noalloc.cu -- mixed-precision charge spreading that allocates nothing.
//
// Who needs this: a caller that may not allocate device memory while it runs
// the spread.  Typical cases are a host simulation engine that owns every
// byte of device memory through its own pool and budget (a foreign
// cudaMalloc would break its accounting or fail outright once the pool has
// taken the free memory), and a time-step loop that cannot afford the
// implicit device-wide synchronisation a cudaMalloc/cudaFree can bring.
// Every other entry point of this library allocates grids and staging
// buffers inside a context; this one only uses memory that exists from the
// moment the library is loaded.
//
// How: the int64 fixed-point accumulation grid that the mixed spread needs
// besides its inputs and output is the file-scope device array below, of a
// fixed size (GSE_NOALLOC_MAX_GRID_POINTS values, 8 MiB).  Every GPU that
// loads the library holds these 8 MiB until the process exits.  The caller
// passes the positions and the output grid in device memory.
#include <cuda.h>

#include <mutex>
#include <vector>

#include "gse_b200.h"
#include "gse_internal.cuh"
#include "gse_kernels.cuh"

namespace gse {
gse_status_t set_error(gse_status_t s, const char* msg);
gse_status_t check_ptr(const void* p, int device, size_t align, const char* what);
}

namespace {

constexpr long long kMaxPoints = GSE_NOALLOC_MAX_GRID_POINTS;

// The scratch grid.  Host code must not use this name as a device address:
// on the host it is only a stand-in symbol.  Its device address is looked up
// once per device with cudaGetSymbolAddress.
static __device__ __align__(256) long long g_noalloc_fixed_grid[kMaxPoints];

// Resolved addresses of the scratch array, one per (device, CUDA context):
// every context that loads the library's device code holds its own copy of
// the array, so a caller that drives its own driver-API contexts gets the
// copy of the context current at the call.
struct ScratchAddr {
  int dev;
  CUcontext ctx;
  long long* ptr;
};
std::vector<ScratchAddr> g_scratch;
std::mutex g_scratch_mu;

// The calling thread's current CUDA context (NULL if none is current yet),
// through the driver entry point the runtime hands out, so that the library
// does not link the driver library itself.
CUcontext current_context() {
  typedef CUresult (*GetCurrentFn)(CUcontext*);
  static const GetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (GetCurrentFn) nullptr;
    }
    return (GetCurrentFn)f;
  }();
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

bool is_device_memory(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

#define TRY_NA(call)                  \
  do {                                \
    gse_status_t _s = (call);         \
    if (_s != GSE_OK) return _s;      \
  } while (0)

}  // namespace

extern "C" gse_status_t gse_spread_mixed_noalloc(int size_x, int size_y, int size_z, double sigma,
                                                 double rcut, int n, const float* xyzq,
                                                 double box_x, double box_y, double box_z,
                                                 float* rho_out, void* stream) {
  using namespace gse;
  if (size_x < 1 || size_y < 1 || size_z < 1)
    return set_error(GSE_ERR_INVALID_ARG, "grid sizes must be >= 1");
  const long long points = (long long)size_x * size_y * size_z;
  if (points > kMaxPoints)
    return set_error(GSE_ERR_INVALID_ARG,
                     "grid exceeds the no-allocation limit of GSE_NOALLOC_MAX_GRID_POINTS "
                     "(1048576) points");
  if (!(sigma > 0.0) || !(rcut > 0.0) || !std::isfinite(sigma) || !std::isfinite(rcut) ||
      !(box_x > 0.0) || !(box_y > 0.0) || !(box_z > 0.0))
    return set_error(GSE_ERR_INVALID_ARG, "sigma, rcut and box lengths must be positive");
  if (n < 0) return set_error(GSE_ERR_INVALID_ARG, "negative atom count");
  const int M[3] = {size_x, size_y, size_z};
  const double box[3] = {box_x, box_y, box_z};
  for (int d = 0; d < 3; d++)
    if (2 * (int)std::ceil(rcut / (box[d] / (double)M[d])) + 1 > kMaxStencil)
      return set_error(GSE_ERR_STENCIL_TOO_LARGE, "stencil wider than 64 points");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
    cudaGetLastError();
    return set_error(GSE_ERR_CUDA, "no current CUDA device");
  }
  if (!rho_out || !is_device_memory(rho_out))
    return set_error(GSE_ERR_INVALID_ARG, "rho_out must be device memory of the current device");
  if (n > 0 && (!xyzq || !is_device_memory(xyzq)))
    return set_error(GSE_ERR_INVALID_ARG, "xyzq must be device memory of the current device");
  // the right device, and the alignment of the kernels' float4 record loads
  TRY_NA(check_ptr(rho_out, dev, sizeof(float), "rho_out"));
  TRY_NA(check_ptr(xyzq, dev, sizeof(float4), "xyzq"));

  // First call on this device (in this CUDA context): resolve the scratch
  // array's device address; later calls reuse it.
  long long* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    CUcontext ctx = current_context();
    for (const ScratchAddr& a : g_scratch)
      if (a.dev == dev && a.ctx == ctx && ctx) scratch = a.ptr;
    if (!scratch) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_fixed_grid);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return set_error(GSE_ERR_CUDA, "cudaGetSymbolAddress of the scratch grid failed");
      }
      scratch = (long long*)p;
      // the lookup makes the runtime's context current if none was
      ctx = current_context();
      if (ctx) g_scratch.push_back({dev, ctx, scratch});
    }
  }

  Stencil<float> s = make_stencil<float>(M, box, sigma, rcut, false, false, 1.0);
  s.fixed_scale = fixed_scale_for((double)s.pref);
  // launch_spread clears the scratch grid, spreads and converts into rho_out
  const cudaError_t e = launch_spread<float>((const float4*)xyzq, n, s, rho_out, scratch,
                                             (cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(GSE_ERR_CUDA, cudaGetErrorString(e));
  return GSE_OK;
}
