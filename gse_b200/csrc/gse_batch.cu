// gse_batch.cu -- many independent GSE-k systems of uneven size, solved
// together (mixed form).
//
// Layout: the caller's atoms of all systems are concatenated (system after
// system).  They are binned with one global key (each system owns a range of
// bins), so after the stable sort every system's atoms are again contiguous
// and in system order.  Real grids and half spectra are grouped by grid size,
// which makes each size class one strided batch for cuFFT.  Spread and gather
// are persistent kernels over a list of (system, brick) work items; the
// Green's-function tables are built once per system in FP64.  The whole
// evaluation (and, if asked, the reverse pass) can be captured into a CUDA
// graph and replayed.  A small autotuner times the persistent-CTA counts and
// the order of the work items on the batch itself and caches the choice.
#include <cufft.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <initializer_list>
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "gse_adjoint.cuh"
#include "gse_b200.h"
#include "gse_internal.cuh"
#include "gse_kernels.cuh"
#include "gse_tiled.cuh"

namespace gse {
gse_status_t set_error(gse_status_t s, const char* msg);
gse_status_t check_ptr(const void* p, int device, size_t align, const char* what);
}

using namespace gse;

namespace {

struct SizeClass {
  int M[3];
  int count;
  long long goff, koff;  // first real point / complex bin of the class
  cufftHandle pf = 0, pb = 0;
};

}  // namespace

struct gse_batch {
  gse_params_t p;
  int nsys = 0, ntot = 0, dev = 0;
  cudaStream_t stream = nullptr;
  std::vector<BatchSys> sys;
  std::vector<int> first;
  std::vector<SizeClass> cls;
  std::vector<BatchItem> scat, gath, agath;  // spread, gather, reverse-pass gather bricks
  std::vector<BatchSeg> scat_seg, gath_seg, agath_seg;  // runs of one stencil width
  int nbins = 0;
  long long gtot = 0, ktot = 0;
  // device
  BatchSys* d_sys = nullptr;
  int* d_first = nullptr;
  long long* d_kfirst = nullptr;
  int* d_ksys = nullptr;
  BatchItem* d_scat = nullptr;
  BatchItem* d_gath = nullptr;
  BatchItem* d_agath = nullptr;
  float4* d_xyzq = nullptr;
  float4* d_sorted = nullptr;
  int* d_perm = nullptr;
  int* d_key = nullptr;
  int* d_tmp = nullptr;
  int* d_counts = nullptr;
  int* d_start = nullptr;
  int* d_tiles = nullptr;
  unsigned* d_qmax = nullptr;
  long long* d_g64 = nullptr;
  float* d_rho = nullptr;
  float* d_phi = nullptr;
  float* d_lam = nullptr;
  float2* d_rhok = nullptr;
  float* d_gtab = nullptr;
  double* d_energy = nullptr;
  double* d_forces = nullptr;  // 3 x ntot
  double* d_dLdE = nullptr;    // nsys
  double* d_gin = nullptr;     // 3 x ntot
  double* d_gout = nullptr;    // 4 x ntot
  int scat_ctas = 0, gath_ctas = 0, agath_ctas = 0;
  bool largest_first = false;
  // one persistent cooperative launch per direction (grids that are multiples
  // of 8 and at most 64 points per side); otherwise the per-stage launches
  bool fused = false, fused_ok = false;
  int fused_ctas = 0, gather_lanes = 16;
  int graph_kernels = 0;  // kernel nodes of the captured graph
  int* d_line_first = nullptr;  // [3][nsys + 1]: x rows, y columns, z columns
  int* d_qctr = nullptr;        // [4] work-item counters of the fused launches
  double* d_epart = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
};

namespace {

#define BCU(call)                                                                       \
  do {                                                                                  \
    cudaError_t _e = (call);                                                            \
    if (_e != cudaSuccess) {                                                            \
      char _m[400];                                                                     \
      snprintf(_m, sizeof(_m), "%s: %s", #call, cudaGetErrorString(_e));                \
      return set_error(_e == cudaErrorMemoryAllocation ? GSE_ERR_OOM : GSE_ERR_CUDA, _m); \
    }                                                                                   \
  } while (0)

#define BFFT(call)                                                                      \
  do {                                                                                  \
    cufftResult _r = (call);                                                            \
    if (_r != CUFFT_SUCCESS) {                                                          \
      char _m[200];                                                                     \
      snprintf(_m, sizeof(_m), "%s: cufft error %d", #call, (int)_r);                   \
      return set_error(GSE_ERR_CUDA, _m);                                               \
    }                                                                                   \
  } while (0)

#define BTRY(call)                     \
  do {                                 \
    gse_status_t _s = (call);          \
    if (_s != GSE_OK) return _s;       \
  } while (0)

// A caller's buffer that is device memory must be on the batch's device; the
// batch only copies into and out of its own buffers, so any alignment does.
gse_status_t check_bufs(int dev, std::initializer_list<const void*> ptrs) {
  for (const void* p : ptrs) BTRY(check_ptr(p, dev, 1, "batch input or output"));
  return GSE_OK;
}

bool is_dev(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Order the work items: natural (system, brick) order or by descending work.
void order_items(gse_batch_t* b, bool largest_first) {
  auto by_work = [&](std::vector<BatchItem>& v) {
    std::stable_sort(v.begin(), v.end(), [&](const BatchItem& x, const BatchItem& y) {
      const int nx = b->sys[x.sys].n, ny = b->sys[y.sys].n;
      return nx > ny;
    });
  };
  std::vector<BatchItem> s, g, ag;
  for (int k = 0; k < b->nsys; k++) {
    const BatchSys& S = b->sys[k];
    const int ns[3] = {(S.b.M[0] + kSB - 1) / kSB, (S.b.M[1] + kSB - 1) / kSB,
                       (S.b.M[2] + kSB - 1) / kSB};
    for (int z = 0; z < ns[2]; z++)
      for (int y = 0; y < ns[1]; y++)
        for (int x = 0; x < ns[0]; x++) s.push_back({k, x, y, z});
    const int ng[3] = {(S.b.M[0] + kGX - 1) / kGX, (S.b.M[1] + kGY - 1) / kGY,
                       (S.b.M[2] + kGZ - 1) / kGZ};
    for (int z = 0; z < ng[2]; z++)
      for (int y = 0; y < ng[1]; y++)
        for (int x = 0; x < ng[0]; x++) g.push_back({k, x, y, z});
    const int na[3] = {(S.b.M[0] + kAX - 1) / kAX, (S.b.M[1] + kAY - 1) / kAY,
                       (S.b.M[2] + kAZ - 1) / kAZ};
    for (int z = 0; z < na[2]; z++)
      for (int y = 0; y < na[1]; y++)
        for (int x = 0; x < na[0]; x++) ag.push_back({k, x, y, z});
  }
  if (largest_first) {
    by_work(s);
    by_work(g);
    by_work(ag);
  }
  // group by stencil width (stable, so the order above holds within a width)
  auto by_width = [&](std::vector<BatchItem>& v, std::vector<BatchSeg>& seg) {
    std::stable_sort(v.begin(), v.end(), [&](const BatchItem& x, const BatchItem& y) {
      return b->sys[x.sys].W < b->sys[y.sys].W;
    });
    seg.clear();
    for (int i = 0; i < (int)v.size(); i++) {
      const int w = b->sys[v[i].sys].W;
      if (seg.empty() || seg.back().W != w) seg.push_back({w, i, 0});
      seg.back().count++;
    }
  };
  by_width(s, b->scat_seg);
  by_width(g, b->gath_seg);
  by_width(ag, b->agath_seg);
  b->scat = s;
  b->gath = g;
  b->agath = ag;
  b->largest_first = largest_first;
}

gse_status_t upload_items(gse_batch_t* b) {
  BCU(cudaMemcpy(b->d_scat, b->scat.data(), sizeof(BatchItem) * b->scat.size(),
                 cudaMemcpyHostToDevice));
  BCU(cudaMemcpy(b->d_gath, b->gath.data(), sizeof(BatchItem) * b->gath.size(),
                 cudaMemcpyHostToDevice));
  BCU(cudaMemcpy(b->d_agath, b->agath.data(), sizeof(BatchItem) * b->agath.size(),
                 cudaMemcpyHostToDevice));
  return GSE_OK;
}

// Arguments of the fused launches on the batch's buffers.
BatchFused fused_args(const gse_batch_t* b) {
  BatchFused a{};
  a.xyzq = b->d_xyzq;
  a.ntot = b->ntot;
  a.nsys = b->nsys;
  a.nbins = b->nbins;
  a.sys = b->d_sys;
  a.first = b->d_first;
  a.w = BinScratch{b->d_key, b->d_counts, b->d_start, b->d_tiles, b->d_tmp, b->d_qmax};
  a.sorted = b->d_sorted;
  a.perm = b->d_perm;
  a.scat = b->d_scat;
  a.nscat = (int)b->scat.size();
  a.gath = b->d_gath;
  a.ngath = (int)b->gath.size();
  a.agath = b->d_agath;
  a.nagath = (int)b->agath.size();
  a.g64 = b->d_g64;
  a.gtot = b->gtot;
  a.rhok = b->d_rhok;
  a.gtab = b->d_gtab;
  a.phi = b->d_phi;
  a.psi = b->d_lam;
  a.qctr = b->d_qctr;
  a.xrow_first = b->d_line_first;
  a.ycol_first = b->d_line_first + (b->nsys + 1);
  a.zcol_first = b->d_line_first + 2 * (b->nsys + 1);
  a.epart = b->d_epart;
  a.energy = b->d_energy;
  a.ccelec = b->p.ccelec;
  a.fx = b->d_forces;
  a.fy = b->d_forces + b->ntot;
  a.fz = b->d_forces + 2 * (long long)b->ntot;
  a.dLdE = b->d_dLdE;
  const long long nt = b->ntot;
  a.gfx = b->d_gin;
  a.gfy = b->d_gin + nt;
  a.gfz = b->d_gin + 2 * nt;
  a.dq = b->d_gout;
  a.dx = b->d_gout + nt;
  a.dy = b->d_gout + 2 * nt;
  a.dz = b->d_gout + 3 * nt;
  return a;
}

// One batched evaluation on the batch's device buffers (all on b->stream).
gse_status_t run_forward(gse_batch_t* b) {
  cudaStream_t st = b->stream;
  if (b->fused) {
    BCU(launch_batch_forward_fused(fused_args(b), b->fused_ctas, b->gather_lanes, st));
    return GSE_OK;
  }
  BinScratch w{b->d_key, b->d_counts, b->d_start, b->d_tiles, b->d_tmp, b->d_qmax};
  BCU(launch_batch_bin(b->d_xyzq, b->ntot, b->d_sys, b->d_first, b->nsys, b->nbins, w,
                       b->d_sorted, b->d_perm, st));
  BCU(launch_batch_spread(b->d_sorted, b->d_start, b->d_sys, b->d_scat, b->scat_seg.data(),
                          (int)b->scat_seg.size(), b->scat_ctas, b->d_g64, b->gtot, b->d_rho, st));
  for (const SizeClass& c : b->cls)
    BFFT(cufftExecR2C(c.pf, (cufftReal*)(b->d_rho + c.goff), (cufftComplex*)(b->d_rhok + c.koff)));
  BCU(cudaMemsetAsync(b->d_energy, 0, sizeof(double) * b->nsys, st));
  BCU(launch_batch_green(b->d_rhok, b->d_gtab, b->ktot, b->d_sys, b->d_kfirst, b->d_ksys, b->nsys,
                         b->d_energy, st));
  for (const SizeClass& c : b->cls)
    BFFT(cufftExecC2R(c.pb, (cufftComplex*)(b->d_rhok + c.koff), (cufftReal*)(b->d_phi + c.goff)));
  BCU(launch_batch_gather(b->d_sorted, b->d_perm, b->d_start, b->d_sys, b->d_gath,
                          b->gath_seg.data(), (int)b->gath_seg.size(), b->gath_ctas, b->d_phi,
                          b->p.ccelec, b->d_forces,
                          b->d_forces + b->ntot, b->d_forces + 2 * (long long)b->ntot, st));
  return GSE_OK;
}

// Reverse pass after run_forward: uses d_dLdE and d_gin, writes d_gout.
gse_status_t run_adjoint(gse_batch_t* b) {
  cudaStream_t st = b->stream;
  if (b->fused) {
    BCU(launch_batch_reverse_fused(fused_args(b), b->fused_ctas, st));
    return GSE_OK;
  }
  const long long nt = b->ntot;
  BCU(launch_batch_adj_scatter(b->d_sorted, b->d_perm, b->d_start, b->d_sys, b->d_scat,
                               b->scat_seg.data(), (int)b->scat_seg.size(), b->scat_ctas,
                               b->p.ccelec, b->d_gin,
                               b->d_gin + nt, b->d_gin + 2 * nt, b->d_g64, b->gtot, b->d_lam, st));
  for (const SizeClass& c : b->cls)
    BFFT(cufftExecR2C(c.pf, (cufftReal*)(b->d_lam + c.goff), (cufftComplex*)(b->d_rhok + c.koff)));
  BCU(launch_batch_green(b->d_rhok, b->d_gtab, b->ktot, b->d_sys, b->d_kfirst, b->d_ksys, b->nsys,
                         nullptr, st));
  for (const SizeClass& c : b->cls)
    BFFT(cufftExecC2R(c.pb, (cufftComplex*)(b->d_rhok + c.koff), (cufftReal*)(b->d_lam + c.goff)));
  BCU(launch_batch_adj_gather_tiled(b->d_sorted, b->d_perm, b->d_start, b->d_sys, b->d_agath,
                                    b->agath_seg.data(), (int)b->agath_seg.size(),
                                    b->agath_ctas, b->p.ccelec, b->d_dLdE, b->d_lam, b->d_phi,
                                    b->d_gin, b->d_gin + nt, b->d_gin + 2 * nt, b->d_gout,
                                    b->d_gout + nt, b->d_gout + 2 * nt, b->d_gout + 3 * nt, st));
  return GSE_OK;
}

gse_status_t set_stream_all(gse_batch_t* b, cudaStream_t st) {
  b->stream = st;
  for (SizeClass& c : b->cls) {
    BFFT(cufftSetStream(c.pf, st));
    BFFT(cufftSetStream(c.pb, st));
  }
  return GSE_OK;
}

gse_status_t drop_graph(gse_batch_t* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->gexec = nullptr;
  b->graph = nullptr;
  return GSE_OK;
}

std::string tune_key(const gse_batch_t* b) {
  std::map<int, int> hist;
  for (const SizeClass& c : b->cls) hist[c.M[0] * 1000000 + c.M[1] * 1000 + c.M[2]] += c.count;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->dev);
  char buf[64];
  std::string k = b->fused_ok ? "batchf" : "batch";
  snprintf(buf, sizeof(buf), "-n%d-N%d-sm%d", b->nsys, (int)std::log2((double)b->ntot + 1), sms);
  k += buf;
  for (auto& kv : hist) {
    snprintf(buf, sizeof(buf), "-%dx%d", kv.first, kv.second);
    k += buf;
  }
  return k;
}

}  // namespace

extern "C" {

gse_status_t gse_batch_create(const gse_params_t* common, int nsys, const gse_system_t* systems,
                              gse_batch_t** out) {
  if (!common || !systems || !out || nsys < 1)
    return set_error(GSE_ERR_INVALID_ARG, "gse_batch_create: bad arguments");
  *out = nullptr;
  if (common->precision != GSE_PRECISION_MIXED)
    return set_error(GSE_ERR_UNSUPPORTED, "batched systems are built for the mixed form");
  if (!(common->kappa >= 0.0 && common->kappa <= 0.5) || !(common->sigma > 0.0))
    return set_error(GSE_ERR_INVALID_ARG, "bad sigma or kappa");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(GSE_ERR_UNSUPPORTED, "no CUDA device");
  }
  BCU(cudaSetDevice(common->device));
  gse_batch_t* b = new gse_batch_t();
  b->p = *common;
  b->dev = common->device;
  b->nsys = nsys;
  const double sigma1 = common->sigma * std::sqrt(common->kappa);
  const double sigma2 = common->sigma * std::sqrt(1.0 - 2.0 * common->kappa);
  const double rcut1 = common->lambda_sigma1 * std::sqrt(2.0) * sigma1;
  // systems, bins and atoms in the caller's order
  b->sys.resize(nsys);
  b->first.assign(nsys + 1, 0);
  int bin_off = 0;
  for (int k = 0; k < nsys; k++) {
    const gse_system_t& y = systems[k];
    if (y.n < 0 || y.size_x < kMinTiledGrid || y.size_y < kMinTiledGrid ||
        y.size_z < kMinTiledGrid || !(y.box_x > 0 && y.box_y > 0 && y.box_z > 0)) {
      delete b;
      return set_error(GSE_ERR_INVALID_ARG, "system: n >= 0, grid sides >= 10, box > 0");
    }
    BatchSys& S = b->sys[k];
    const int M[3] = {y.size_x, y.size_y, y.size_z};
    const double box[3] = {y.box_x, y.box_y, y.box_z};
    S.b = make_bin_layout(M, kBinX32);
    S.bin_off = bin_off;
    if ((long long)bin_off + bin_count(S.b) > 4096LL * 4096LL) {
      delete b;
      return set_error(GSE_ERR_INVALID_ARG, "batch too large: more than 2^24 atom bins");
    }
    bin_off += bin_count(S.b);
    S.atom_off = b->first[k];
    S.n = y.n;
    b->first[k + 1] = b->first[k] + y.n;
    S.sp = make_stencil<float>(M, box, sigma1, rcut1, false, false, 1.0);
    S.sg = make_stencil<float>(M, box, sigma1, rcut1, true, false, 1.0);
    if (!spread_tiled_supported<float>(S.sp)) {
      delete b;
      return set_error(GSE_ERR_UNSUPPORTED, "stencil width must be 9, 11, 13 or 15 on every axis");
    }
    S.W = 2 * S.sp.nst[0] + 1;
    const double h3 = (box[0] / M[0]) * (box[1] / M[1]) * (box[2] / M[2]);
    S.h3 = h3;
    S.efac = 0.5 * common->ccelec * h3;
  }
  b->nbins = bin_off;
  b->ntot = b->first[nsys];
  // grids grouped by size
  std::map<long long, std::vector<int>> bysize;
  for (int k = 0; k < nsys; k++) {
    const BatchSys& S = b->sys[k];
    bysize[((long long)S.b.M[2] * 4096 + S.b.M[1]) * 4096 + S.b.M[0]].push_back(k);
  }
  std::vector<long long> kf;
  std::vector<int> ks;
  long long go = 0, ko = 0;
  for (auto& kv : bysize) {
    SizeClass c;
    const BatchSys& S0 = b->sys[kv.second[0]];
    for (int d = 0; d < 3; d++) c.M[d] = S0.b.M[d];
    c.count = (int)kv.second.size();
    c.goff = go;
    c.koff = ko;
    const long long gp = (long long)c.M[0] * c.M[1] * c.M[2];
    const long long kp = (long long)(c.M[0] / 2 + 1) * c.M[1] * c.M[2];
    for (int k : kv.second) {
      b->sys[k].grid_off = go;
      b->sys[k].kgrid_off = ko;
      kf.push_back(ko);
      ks.push_back(k);
      go += gp;
      ko += kp;
    }
    b->cls.push_back(c);
  }
  b->gtot = go;
  b->ktot = ko;
  kf.push_back(ko);
  auto bail = [&](gse_status_t s) {
    gse_batch_destroy(b);
    return s;
  };
#define BCUC(call)                                                                        \
  do {                                                                                    \
    cudaError_t _e = (call);                                                              \
    if (_e != cudaSuccess)                                                                \
      return bail(set_error(_e == cudaErrorMemoryAllocation ? GSE_ERR_OOM : GSE_ERR_CUDA, \
                            cudaGetErrorString(_e)));                                     \
  } while (0)
  const size_t na = std::max(b->ntot, 1);
  BCUC(cudaMalloc(&b->d_sys, sizeof(BatchSys) * nsys));
  BCUC(cudaMemcpy(b->d_sys, b->sys.data(), sizeof(BatchSys) * nsys, cudaMemcpyHostToDevice));
  BCUC(cudaMalloc(&b->d_first, sizeof(int) * (nsys + 1)));
  BCUC(cudaMemcpy(b->d_first, b->first.data(), sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice));
  BCUC(cudaMalloc(&b->d_kfirst, sizeof(long long) * kf.size()));
  BCUC(cudaMemcpy(b->d_kfirst, kf.data(), sizeof(long long) * kf.size(), cudaMemcpyHostToDevice));
  BCUC(cudaMalloc(&b->d_ksys, sizeof(int) * ks.size()));
  BCUC(cudaMemcpy(b->d_ksys, ks.data(), sizeof(int) * ks.size(), cudaMemcpyHostToDevice));
  BCUC(cudaMalloc(&b->d_xyzq, sizeof(float4) * na));
  BCUC(cudaMalloc(&b->d_sorted, sizeof(float4) * na));
  BCUC(cudaMalloc(&b->d_perm, sizeof(int) * na));
  BCUC(cudaMalloc(&b->d_key, sizeof(int) * na));
  BCUC(cudaMalloc(&b->d_tmp, sizeof(int) * na));
  BCUC(cudaMalloc(&b->d_counts, sizeof(int) * b->nbins));
  BCUC(cudaMalloc(&b->d_start, sizeof(int) * (b->nbins + 1)));
  BCUC(cudaMalloc(&b->d_tiles, sizeof(int) * (b->nbins / 4096 + 2)));
  BCUC(cudaMalloc(&b->d_qmax, sizeof(unsigned)));
  BCUC(cudaMalloc(&b->d_g64, sizeof(long long) * b->gtot));
  BCUC(cudaMalloc(&b->d_rho, sizeof(float) * b->gtot));
  BCUC(cudaMalloc(&b->d_phi, sizeof(float) * b->gtot));
  BCUC(cudaMalloc(&b->d_lam, sizeof(float) * b->gtot));
  BCUC(cudaMalloc(&b->d_rhok, sizeof(float2) * b->ktot));
  BCUC(cudaMalloc(&b->d_gtab, sizeof(float) * b->ktot));
  BCUC(cudaMalloc(&b->d_energy, sizeof(double) * nsys));
  BCUC(cudaMalloc(&b->d_dLdE, sizeof(double) * nsys));
  BCUC(cudaMalloc(&b->d_forces, sizeof(double) * 3 * na));
  BCUC(cudaMalloc(&b->d_gin, sizeof(double) * 3 * na));
  BCUC(cudaMalloc(&b->d_gout, sizeof(double) * 4 * na));
  BCUC(cudaMemset(b->d_gin, 0, sizeof(double) * 3 * na));
  BCUC(cudaMemset(b->d_dLdE, 0, sizeof(double) * nsys));
  // Green's tables (FP64 arithmetic, stored as float)
  for (int k = 0; k < nsys; k++) {
    const gse_system_t& y = systems[k];
    GreenGeom g;
    g.nfft[0] = y.size_x;
    g.nfft[1] = y.size_y;
    g.nfft[2] = y.size_z;
    for (int d = 0; d < 3; d++) g.half[d] = g.nfft[d] / 2 + (g.nfft[d] % 2);
    g.sizeX = g.nfft[0] / 2 + 1;
    g.nx_even = (g.nfft[0] % 2) == 0;
    g.want_energy = 0;
    g.twopi_box[0] = 2.0 * kPi / y.box_x;
    g.twopi_box[1] = 2.0 * kPi / y.box_y;
    g.twopi_box[2] = 2.0 * kPi / y.box_z;
    g.fourpi_vol = 4.0 * kPi / (double)(g.nfft[0] * g.nfft[1] * g.nfft[2]);
    g.sigmafac = sigma2 * sigma2 / 2.0;
    BCUC(launch_green_table<float>(g, b->d_gtab + b->sys[k].kgrid_off, nullptr));
  }
  // cuFFT: one strided batch per size class
  for (SizeClass& c : b->cls) {
    int nn[3] = {c.M[2], c.M[1], c.M[0]};
    const int gp = c.M[0] * c.M[1] * c.M[2], kp = (c.M[0] / 2 + 1) * c.M[1] * c.M[2];
    if (cufftPlanMany(&c.pf, 3, nn, nullptr, 1, gp, nullptr, 1, kp, CUFFT_R2C, c.count) !=
            CUFFT_SUCCESS ||
        cufftPlanMany(&c.pb, 3, nn, nullptr, 1, kp, nullptr, 1, gp, CUFFT_C2R, c.count) !=
            CUFFT_SUCCESS)
      return bail(set_error(GSE_ERR_CUDA, "cufftPlanMany failed"));
  }
  const int sms = sm_count();
  b->scat_ctas = 2 * sms;
  b->gath_ctas = 2 * sms;
  b->agath_ctas = 2 * sms;
  // the fused launches are available when every grid side is a multiple of 8
  // and at most 64 and the cooperative grid can be resident
  // (GSE_B200_BATCH_FUSED=0 withholds them); the batch starts on the per-stage
  // launches, the autotuner or gse_batch_set_schedule may switch
  {
    const char* env = getenv("GSE_B200_BATCH_FUSED");
    const bool allowed = !(env && env[0] == '0');
    const int fc = std::min(batch_fused_ctas(16), batch_fused_rev_ctas());
    if (allowed && fc > 0 && batch_fused_supported(b->sys.data(), nsys)) {
      // line counts of the FFT passes: x rows My Mz, y columns Mz Hx, z columns My Hx
      std::vector<int> lf(3 * (nsys + 1), 0);
      for (int k = 0; k < nsys; k++) {
        const int* M = b->sys[k].b.M;
        const int hx = M[0] / 2 + 1;
        lf[k + 1] = lf[k] + M[1] * M[2];
        lf[(nsys + 1) + k + 1] = lf[(nsys + 1) + k] + M[2] * hx;
        lf[2 * (nsys + 1) + k + 1] = lf[2 * (nsys + 1) + k] + M[1] * hx;
      }
      BCUC(cudaMalloc(&b->d_line_first, sizeof(int) * lf.size()));
      BCUC(cudaMemcpy(b->d_line_first, lf.data(), sizeof(int) * lf.size(),
                      cudaMemcpyHostToDevice));
      BCUC(cudaMalloc(&b->d_epart, sizeof(double) * std::max(lf[3 * (nsys + 1) - 1], 1)));
      BCUC(cudaMalloc(&b->d_qctr, sizeof(int) * 4));
      BCUC(cudaMemset(b->d_qctr, 0, sizeof(int) * 4));
      b->fused_ok = true;
      b->fused_ctas = fc;
      b->gather_lanes = 16;
    }
    cudaGetLastError();
  }
  order_items(b, true);
  BCUC(cudaMalloc(&b->d_scat, sizeof(BatchItem) * std::max<size_t>(b->scat.size(), 1)));
  BCUC(cudaMalloc(&b->d_gath, sizeof(BatchItem) * std::max<size_t>(b->gath.size(), 1)));
  BCUC(cudaMalloc(&b->d_agath, sizeof(BatchItem) * std::max<size_t>(b->agath.size(), 1)));
  if (upload_items(b) != GSE_OK) return bail(GSE_ERR_CUDA);
  BCUC(cudaDeviceSynchronize());
#undef BCUC
  *out = b;
  return GSE_OK;
}

gse_status_t gse_batch_destroy(gse_batch_t* b) {
  if (!b) return GSE_OK;
  cudaSetDevice(b->dev);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (SizeClass& c : b->cls) {
    if (c.pf) cufftDestroy(c.pf);
    if (c.pb) cufftDestroy(c.pb);
  }
  void* ptrs[] = {b->d_line_first, b->d_epart, b->d_qctr,
                  b->d_sys, b->d_first, b->d_kfirst, b->d_ksys, b->d_scat, b->d_gath, b->d_agath,
                  b->d_xyzq, b->d_sorted, b->d_perm, b->d_key, b->d_tmp, b->d_counts,
                  b->d_start, b->d_tiles, b->d_qmax, b->d_g64, b->d_rho, b->d_phi, b->d_lam,
                  b->d_rhok, b->d_gtab, b->d_energy, b->d_dLdE, b->d_forces, b->d_gin,
                  b->d_gout};
  for (void* q : ptrs) cudaFree(q);
  delete b;
  return GSE_OK;
}

gse_status_t gse_batch_set_stream(gse_batch_t* b, void* stream) {
  if (!b) return set_error(GSE_ERR_INVALID_ARG, "NULL batch");
  BCU(cudaSetDevice(b->dev));
  drop_graph(b);
  return set_stream_all(b, (cudaStream_t)stream);
}

gse_status_t gse_batch_info(gse_batch_t* b, gse_batch_info_t* info) {
  if (!b || !info) return set_error(GSE_ERR_INVALID_ARG, "NULL argument");
  info->n_total = b->ntot;
  info->n_systems = b->nsys;
  info->n_size_classes = (int)b->cls.size();
  info->grid_points = b->gtot;
  info->scatter_items = (int)b->scat.size();
  info->gather_items = (int)b->gath.size();
  info->scatter_ctas = b->scat_ctas;
  info->gather_ctas = b->gath_ctas;
  info->largest_first = b->largest_first ? 1 : 0;
  info->xyzq = b->d_xyzq;
  info->energies = b->d_energy;
  info->forces = b->d_forces;
  info->dLdE = b->d_dLdE;
  info->grad_forces = b->d_gin;
  info->grad_out = b->d_gout;
  info->fused = b->fused ? 1 : 0;
  info->fused_available = b->fused_ok ? 1 : 0;
  info->gather_lanes = b->fused ? b->gather_lanes : kGatherLanes;
  info->fused_ctas = b->fused ? b->fused_ctas : 0;
  info->graph_kernels = b->gexec ? b->graph_kernels : 0;
  return GSE_OK;
}

gse_status_t gse_batch_forward(gse_batch_t* b, const void* xyzq, double* energies, double* fx,
                               double* fy, double* fz) {
  if (!b) return set_error(GSE_ERR_INVALID_ARG, "NULL batch");
  BTRY(check_bufs(b->dev, {xyzq, energies, fx, fy, fz}));
  BCU(cudaSetDevice(b->dev));
  cudaStream_t st = b->stream;
  if (xyzq && xyzq != (const void*)b->d_xyzq && b->ntot > 0)
    BCU(cudaMemcpyAsync(b->d_xyzq, xyzq, sizeof(float4) * b->ntot,
                        is_dev(xyzq) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  BTRY(run_forward(b));
  bool host = false;
  auto out = [&](void* dst, const void* src, size_t bytes) -> gse_status_t {
    if (!dst || dst == src) return GSE_OK;
    const bool d = is_dev(dst);
    if (!d) host = true;
    BCU(cudaMemcpyAsync(dst, src, bytes, d ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        st));
    return GSE_OK;
  };
  const size_t nb = sizeof(double) * b->ntot;
  BTRY(out(energies, b->d_energy, sizeof(double) * b->nsys));
  BTRY(out(fx, b->d_forces, nb));
  BTRY(out(fy, b->d_forces + b->ntot, nb));
  BTRY(out(fz, b->d_forces + 2 * (long long)b->ntot, nb));
  if (host) BCU(cudaStreamSynchronize(st));
  BCU(cudaGetLastError());
  return GSE_OK;
}

gse_status_t gse_batch_adjoint(gse_batch_t* b, const void* xyzq, const double* dLdE,
                               const double* gfx, const double* gfy, const double* gfz,
                               double* dq, double* dx, double* dy, double* dz) {
  if (!b) return set_error(GSE_ERR_INVALID_ARG, "NULL batch");
  BTRY(check_bufs(b->dev, {xyzq, dLdE, gfx, gfy, gfz, dq, dx, dy, dz}));
  BCU(cudaSetDevice(b->dev));
  cudaStream_t st = b->stream;
  const long long nt = b->ntot;
  auto in = [&](void* dst, const void* src, size_t bytes) -> gse_status_t {
    if (!src || src == dst || bytes == 0) return GSE_OK;
    BCU(cudaMemcpyAsync(dst, src, bytes,
                        is_dev(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    return GSE_OK;
  };
  BTRY(in(b->d_xyzq, xyzq, sizeof(float4) * nt));
  if (dLdE)
    BTRY(in(b->d_dLdE, dLdE, sizeof(double) * b->nsys));
  else
    BCU(cudaMemsetAsync(b->d_dLdE, 0, sizeof(double) * b->nsys, st));
  if (gfx && gfy && gfz) {
    BTRY(in(b->d_gin, gfx, sizeof(double) * nt));
    BTRY(in(b->d_gin + nt, gfy, sizeof(double) * nt));
    BTRY(in(b->d_gin + 2 * nt, gfz, sizeof(double) * nt));
  } else if (gfx || gfy || gfz) {
    return set_error(GSE_ERR_INVALID_ARG, "force gradients: give all three or none");
  } else {
    BCU(cudaMemsetAsync(b->d_gin, 0, sizeof(double) * 3 * nt, st));
  }
  BTRY(run_forward(b));
  BTRY(run_adjoint(b));
  bool host = false;
  double* outs[4] = {dq, dx, dy, dz};
  for (int k = 0; k < 4; k++) {
    if (!outs[k]) continue;
    const bool d = is_dev(outs[k]);
    if (!d) host = true;
    BCU(cudaMemcpyAsync(outs[k], b->d_gout + k * nt, sizeof(double) * nt,
                        d ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  }
  if (host) BCU(cudaStreamSynchronize(st));
  BCU(cudaGetLastError());
  return GSE_OK;
}

gse_status_t gse_batch_capture(gse_batch_t* b, int with_adjoint) {
  if (!b) return set_error(GSE_ERR_INVALID_ARG, "NULL batch");
  BCU(cudaSetDevice(b->dev));
  drop_graph(b);
  // capture needs a stream other than the legacy default stream
  cudaStream_t old = b->stream;
  cudaStream_t cap = old;
  bool own = false;
  if (!cap) {
    BCU(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    own = true;
    BTRY(set_stream_all(b, cap));
  }
  BCU(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
  gse_status_t s = run_forward(b);
  if (s == GSE_OK && with_adjoint) s = run_adjoint(b);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(cap, &g);
  if (s == GSE_OK && e != cudaSuccess)
    s = set_error(GSE_ERR_CUDA, cudaGetErrorString(e));
  if (s == GSE_OK) {
    const cudaError_t ei = cudaGraphInstantiate(&b->gexec, g, 0);
    if (ei != cudaSuccess) s = set_error(GSE_ERR_CUDA, cudaGetErrorString(ei));
  }
  // kernel nodes of the captured graph (library FFT kernels included)
  b->graph_kernels = 0;
  if (s == GSE_OK) {
    size_t nn = 0;
    if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn > 0) {
      std::vector<cudaGraphNode_t> nodes(nn);
      if (cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess)
        for (size_t i = 0; i < nn; i++) {
          cudaGraphNodeType t;
          if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
            b->graph_kernels++;
        }
    }
    cudaGetLastError();
  }
  b->graph = g;
  if (own) {
    set_stream_all(b, old);
    cudaStreamDestroy(cap);
  }
  if (s != GSE_OK) drop_graph(b);
  return s;
}

gse_status_t gse_batch_launch(gse_batch_t* b) {
  if (!b) return set_error(GSE_ERR_INVALID_ARG, "NULL batch");
  if (!b->gexec) return set_error(GSE_ERR_NOT_READY, "no captured graph (gse_batch_capture)");
  BCU(cudaSetDevice(b->dev));
  BCU(cudaGraphLaunch(b->gexec, b->stream));
  return GSE_OK;
}

gse_status_t gse_batch_set_schedule(gse_batch_t* b, int fused, int gather_lanes,
                                    int largest_first, int scatter_ctas, int gather_ctas) {
  if (!b) return set_error(GSE_ERR_INVALID_ARG, "NULL batch");
  if (fused && !b->fused_ok)
    return set_error(GSE_ERR_UNSUPPORTED,
                     "the fused launch needs every grid side a multiple of 8 and at most 64");
  if (fused && gather_lanes != 8 && gather_lanes != 16)
    return set_error(GSE_ERR_INVALID_ARG, "gather lanes per atom must be 8 or 16");
  if (!fused && (scatter_ctas < 1 || gather_ctas < 1))
    return set_error(GSE_ERR_INVALID_ARG, "persistent CTA counts must be positive");
  BCU(cudaSetDevice(b->dev));
  b->fused = fused != 0;
  if (b->fused) {
    b->gather_lanes = gather_lanes;
    b->fused_ctas = std::min(batch_fused_ctas(gather_lanes), batch_fused_rev_ctas());
  } else {
    b->scat_ctas = scatter_ctas;
    b->gath_ctas = gather_ctas;
    b->agath_ctas = gather_ctas;
  }
  order_items(b, largest_first != 0);
  drop_graph(b);
  return upload_items(b);
}

gse_status_t gse_batch_autotune(gse_batch_t* b, const char* cache_path, int use_cache) {
  if (!b) return set_error(GSE_ERR_INVALID_ARG, "NULL batch");
  BCU(cudaSetDevice(b->dev));
  const std::string key = tune_key(b);
  // cached choice?  One line per key: lf fused gl sc gc ms
  if (use_cache && cache_path) {
    FILE* f = fopen(cache_path, "r");
    if (f) {
      char k[512];
      int lf, fu, gl, sc, gc;
      double ms;
      bool found = false;
      while (fscanf(f, "%511s %d %d %d %d %d %lf", k, &lf, &fu, &gl, &sc, &gc, &ms) == 7)
        if (key == k && (!fu || b->fused_ok)) {
          found = true;
          BTRY(gse_batch_set_schedule(b, fu, gl, lf, sc, gc));
        }
      fclose(f);
      if (found) return GSE_OK;
    }
  }
  // every schedule on a forward and a reverse pass of the batch's current
  // inputs: the per-stage launches (work-item order x persistent CTAs of the
  // spread and gather kernels) and, where the grids allow it, the fused
  // launches (work-item order x lanes per atom of the gather)
  struct Cand {
    int lf, fused, gl, sc, gc;
  };
  std::vector<Cand> cands;
  const int sms = sm_count();
  for (int lf = 0; lf < 2; lf++) {
    for (int sc : {sms, 2 * sms})
      for (int gc : {sms, 2 * sms, 4 * sms}) cands.push_back({lf, 0, kGatherLanes, sc, gc});
    if (b->fused_ok)
      for (int gl : {16, 8})
        if (batch_fused_ctas(gl) > 0) cands.push_back({lf, 1, gl, 2 * sms, 2 * sms});
  }
  cudaEvent_t e0, e1;
  BCU(cudaEventCreate(&e0));
  BCU(cudaEventCreate(&e1));
  double best = 1e30;
  Cand bc = cands[0];
  gse_status_t st = GSE_OK;
  for (const Cand& c : cands) {
    st = gse_batch_set_schedule(b, c.fused, c.gl, c.lf, c.sc, c.gc);
    if (st != GSE_OK) break;
    if ((st = run_forward(b)) != GSE_OK || (st = run_adjoint(b)) != GSE_OK) break;  // warm
    cudaEventRecord(e0, b->stream);
    for (int r = 0; r < 3 && st == GSE_OK; r++) {
      st = run_forward(b);
      if (st == GSE_OK) st = run_adjoint(b);
    }
    cudaEventRecord(e1, b->stream);
    if (st != GSE_OK) break;
    float ms = 0.f;
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
      st = set_error(GSE_ERR_CUDA, "autotune timing failed");
      break;
    }
    if (ms / 3.0 < best) {
      best = ms / 3.0;
      bc = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != GSE_OK) return st;
  BTRY(gse_batch_set_schedule(b, bc.fused, bc.gl, bc.lf, bc.sc, bc.gc));
  if (cache_path) {
    FILE* f = fopen(cache_path, "a");
    if (f) {
      fprintf(f, "%s %d %d %d %d %d %.6f\n", key.c_str(), bc.lf, bc.fused, bc.gl, bc.sc, bc.gc,
              best);
      fclose(f);
    }
  }
  return GSE_OK;
}

}  // extern "C"
