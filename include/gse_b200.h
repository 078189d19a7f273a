/*
 * gse_b200.h -- C ABI of the B200-native GSE-k reciprocal-space library.
 *
 * The library computes Gaussian-Split-Ewald k-space electrostatics on one
 * NVIDIA B200 (sm_100a): Gaussian charge spreading onto a periodic grid, the
 * k-space Green's-function multiply around a 3-D real FFT, the mesh energy,
 * and the Gaussian gather of forces.  Every entry point below replaces one
 * public method of the reference classes of ap-hynninen/GSE (paths relative
 * to that project); the C++ drop-in classes in gse_b200/cxx/ and the Python
 * mirror in gse_b200/gse.py forward to these functions.
 *
 * Conventions
 *  - Every call returns a gse_status_t; GSE_OK is 0.  The library never
 *    calls exit() or abort().  gse_last_error() describes the last failure
 *    on the calling thread.
 *  - Grids are x-fastest, index x + (y + z*size_y)*size_x, periodic, as
 *    Grid<T>::getPos (Grid.h:32-44).
 *  - Positions/charges are AoS records {x, y, z, q} of the calculation type
 *    CT: double for GSE_PRECISION_FP64 (xyzq_t<double>), float for
 *    GSE_PRECISION_MIXED (xyzq_t<float>) (TypesGSE.h:19-22).
 *  - Forces and energies are double (the accumulation type AT of both
 *    reference instances <double,double> and <double,float>).
 *  - A pointer argument may be host memory (pageable or pinned) or device
 *    memory of the context's device; the library inspects it.  Calls whose
 *    outputs are host memory return after the results are written; calls
 *    whose outputs are all device memory are asynchronous on the context's
 *    stream.
 *  - A context is not re-entrant: calls on one context must not overlap.
 *    Independent contexts may be used from different threads.
 */
#ifndef GSE_B200_H
#define GSE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define GSE_B200_ABI_VERSION 1

typedef enum gse_status {
  GSE_OK = 0,
  GSE_ERR_INVALID_ARG = 1,       /* bad size, NULL pointer, kappa outside [0, 0.5] ... */
  GSE_ERR_STENCIL_TOO_LARGE = 2, /* 2n+1 > grid size along an axis */
  GSE_ERR_CUDA = 3,              /* a CUDA runtime / cuFFT call failed */
  GSE_ERR_OOM = 4,               /* device or pinned allocation failed */
  GSE_ERR_TIMEOUT = 5,           /* a bounded device-side wait gave up */
  GSE_ERR_NOT_READY = 6,         /* stage called out of order (e.g. energy before solve) */
  GSE_ERR_UNSUPPORTED = 7,       /* no GPU, wrong architecture, or feature not built */
  GSE_ERR_NONFINITE = 8,         /* a position or charge is NaN/Inf: returned by the call
                                    that saw it when its outputs are host memory, else by
                                    the next gse_synchronize (results are then undefined) */
  GSE_ERR_RANGE = 9              /* mixed form: the charge of one 16^3-cell brick exceeds
                                    the int32 tile's fixed-point range: sum over the brick
                                    of |q| (2 pi sigma1^2)^-1.5 above 2^19 (~1.7e7 e at
                                    sigma1 1.26) or one charge's above 2^11 (~6.5e4 e);
                                    reported like GSE_ERR_NONFINITE, results undefined */
} gse_status_t;

typedef enum gse_precision {
  /* plain form: FP64 everywhere (CpuGSEk<double,double>) */
  GSE_PRECISION_FP64 = 0,
  /* mixed form: FP32 positions, stencils and FFT; deterministic int64
   * fixed-point grid accumulation; FP64 Green's-function factors, energy
   * reduction and force accumulation output (CpuGSEk<double,float>) */
  GSE_PRECISION_MIXED = 1
} gse_precision_t;

typedef enum gse_grid_id {
  GSE_GRID_RHO = 0, /* rhoS: spread charge density (CpuGSE::getRhoS, CpuGSE.h:63) */
  GSE_GRID_PHI = 1  /* phiM: mesh potential (CpuGSE::getPhi, CpuGSE.h:64) */
} gse_grid_id_t;

typedef struct gse_params {
  int size_x, size_y, size_z; /* grid points per side (sizeX/Y/Z) */
  double sigma;               /* total Gaussian width */
  double kappa;               /* split: sigma1 = sigma sqrt(kappa), sigma2 = sigma sqrt(1-2 kappa) */
  double lambda_sigma;        /* kept for API parity (CpuGSE.h:52-54); unused by GSE-k */
  double lambda_sigma1;       /* gather/spread cut-off rcut = lambda_sigma1 sqrt(2) sigma1 */
  double box_x, box_y, box_z; /* orthorhombic box lengths */
  double ccelec;              /* unit conversion, CHARMM 332.0716 by default */
  int precision;              /* gse_precision_t */
  int device;                 /* CUDA device ordinal */
} gse_params_t;

typedef struct gse_context gse_context_t;

/* Fill *p with the reference drivers' defaults: kappa 0.4, lambda_sigma and
 * lambda_sigma1 3.0, ccelec 332.0716 (cpu_gse.cpp:424-426, CpuGSE.h:55),
 * FP64 precision, device 0.  Sizes, sigma and box must still be set. */
void gse_params_default(gse_params_t* p);

const char* gse_status_string(gse_status_t s);

/* Text of the last error raised on the calling thread ("" if none). */
const char* gse_last_error(void);

int gse_abi_version(void);

/* Build record of the loaded library: "sources <hash>, nvcc <version>,
 * sm_100a", <hash> the first 16 hex digits of a SHA-256 over the sources it
 * was compiled from (the loader rebuilds a library whose hash differs from
 * the sources beside it). */
const char* gse_build_info(void);

/* ---- context lifetime ------------------------------------------------- */

/* Replaces the constructors CpuGSE(...) / CpuGSEk(...) (CpuGSE.cpp:11-19,
 * CpuGSEk.cpp:14-22) including CpuGSE::setParam's kappa check
 * (CpuGSE.cpp:33-44; the reference asserts, this returns
 * GSE_ERR_INVALID_ARG).  Allocates the grids and FFT plans on the device. */
gse_status_t gse_create(const gse_params_t* params, gse_context_t** out);

/* Replaces ~CpuGSEk / ~CpuFFTSolver (CpuFFTSolver.cpp:18-21). */
gse_status_t gse_destroy(gse_context_t* ctx);

/* Run all following work of this context on `cuda_stream` (a cudaStream_t;
 * NULL selects the legacy default stream). */
gse_status_t gse_set_stream(gse_context_t* ctx, void* cuda_stream);

/* Replaces CpuGSE::setBoxSize (CpuGSE.cpp:58-64). */
gse_status_t gse_set_box(gse_context_t* ctx, double box_x, double box_y, double box_z);

/* Block until the context's queued work has finished. */
gse_status_t gse_synchronize(gse_context_t* ctx);

/* ---- CpuGSEk method equivalents ---------------------------------------- */

/* CpuGSEk::spreadCharge1 (CpuGSEk.cpp:30-33): spread the n charges with
 * sigma1 and rcut1 onto the context's rhoS grid (cleared first). */
gse_status_t gse_spread_charge(gse_context_t* ctx, int n, const void* xyzq);

/* CpuGSEk::solvePoisson (CpuGSEk.cpp:48-50) = CpuFFTSolver::run
 * (CpuFFTSolver.cpp:75-96): phiM = c2r( G(sigma2) * r2c(rhoS) ). */
gse_status_t gse_solve_poisson(gse_context_t* ctx);

/* CpuGSEk::calculateEnergy (CpuGSEk.cpp:56-58, CpuGSE.cpp:86-103):
 * 1/2 ccelec hx hy hz sum rhoS*phiM.  `energy` may be host or device. */
gse_status_t gse_calculate_energy(gse_context_t* ctx, double* energy);

/* CpuGSE::interpolateForce (CpuGSE.cpp:70-80): gather with sigma1 and a
 * spherical cut rcut1 from phiM, times ccelec.  Outputs are overwritten. */
gse_status_t gse_interpolate_force(gse_context_t* ctx, int n, const void* xyzq, double* fx,
                                   double* fy, double* fz);

/* The electric field at the atoms from phiM (after gse_solve_poisson or
 * gse_forward): the gather of interpolateForce (CpuGSE.cpp:70-80,
 * CpuGaussCharge.cpp:105-172, the loop the reference shares between force and
 * field) with every charge taken as 1, i.e. the force per unit charge, times
 * ccelec; defined for neutral sites too.  The charges in xyzq are ignored.
 * Outputs are overwritten. */
gse_status_t gse_interpolate_field(gse_context_t* ctx, int n, const void* xyzq, double* ex,
                                   double* ey, double* ez);

/* One whole force evaluation: spreadCharge1 -> solvePoisson ->
 * calculateEnergy -> interpolateForce, as cpu_gse runs them
 * (cpu_gse.cpp:440-455).  `energy` and the force arrays may be NULL to skip
 * them. */
gse_status_t gse_forward(gse_context_t* ctx, int n, const void* xyzq, double* energy, double* fx,
                         double* fy, double* fz);

/* Copy the rhoS or phiM grid (CT elements, size_x*size_y*size_z) out to
 * host or device memory (CpuGSE::getRhoS / getPhi, CpuGSE.h:63-64). */
gse_status_t gse_get_grid(gse_context_t* ctx, int which, void* out);

/* Load a grid into the context (e.g. a potential to gather from). */
gse_status_t gse_set_grid(gse_context_t* ctx, int which, const void* in);

/* ---- stage entry points with explicit parameters ------------------------ */

/* CpuGaussCharge<AT,CT>::spreadChargeToGrid (CpuGaussCharge.cpp:235-384):
 * full (2n+1)^3 cube, n = ceil(rcut/h), weights exp(-d^2/(2 sigma^2)),
 * prefactor (2 pi sigma^2)^(-3/2); with normalize != 0 each 1-D weight row
 * is rescaled to sum to sqrt(2 pi sigma^2).  rho_out (CT, host or device)
 * receives the grid; the context's rhoS is also updated. */
gse_status_t gse_gauss_spread(gse_context_t* ctx, double sigma, double rcut, int n,
                              const void* xyzq, double box_x, double box_y, double box_z,
                              int normalize, void* rho_out);

/* CpuGaussCharge<AT,CT>::interpolateForce (CpuGaussCharge.cpp:105-183):
 * sum over grid points with r^2 < rcut^2 of
 * q (2 pi)^(-3/2) h^3 sigma^(-5) exp(-r^2/(2 sigma^2)) phi (x - x_p), without
 * the ccelec factor.  phi (CT) may be host or device. */
gse_status_t gse_gauss_interpolate(gse_context_t* ctx, double sigma, double rcut, int n,
                                   const void* xyzq, double box_x, double box_y, double box_z,
                                   const void* phi, double* fx, double* fy, double* fz);

/* CpuGreensFuncGSE<T>::mul (CpuGreensFuncGSE.cpp:9-57), in place on an
 * interleaved complex half spectrum of ((size_x/2+1)*2) x size_y x size_z CT
 * values (host or device). */
gse_status_t gse_green_mul(gse_context_t* ctx, double sigma, double box_x, double box_y,
                           double box_z, void* rho_k);

/* CpuFFTSolver<T>::run (CpuFFTSolver.cpp:75-96) with the GSE Green's
 * function: phi = c2r(G(sigma) r2c(rho)).  rho and phi are CT grids. */
gse_status_t gse_fft_solve(gse_context_t* ctx, double sigma, double box_x, double box_y,
                           double box_z, const void* rho, void* phi);

/* ---- grid operations beside the force path ------------------------------ */

/* CpuGaussCharge<AT,CT>::spreadChargeOnGrid (CpuGaussCharge.cpp:390-519), the
 * second spreading step of the real-space variant (CpuGSEr::spreadCharge2,
 * CpuGSEr.cpp:39-42): rho_s = rho convolved with the periodic Gaussian of
 * width sigma, as three 1-D passes x -> y -> z with taps
 * exp(-h^2 i^2 / (2 sigma^2)), i = -n..n, n = ceil(rcut / h), the z taps
 * times (2 pi sigma^2)^(-3/2) hx hy hz.  Bit-identical to the reference in
 * both calculation types.  rho and rho_s are CT grids of the context's size
 * (host or device; the same device grid may be passed for both).  A host
 * rho_s also leaves the result in the context's rhoS. */
gse_status_t gse_gauss_spread_on_grid(gse_context_t* ctx, double sigma, double rcut,
                                      double box_x, double box_y, double box_z, const void* rho,
                                      void* rho_s);

/* CpuGaussCharge<AT,CT>::calcElectricFieldOnGrid (CpuGaussCharge.cpp:62-98):
 * E_d(p) = -(phi(p + e_d) - phi(p)) / h_d, periodic, in CT (bit-identical to
 * the reference).  phi, ex, ey, ez are CT grids of the context's size (host or
 * device); phi must not be one of the outputs. */
gse_status_t gse_gauss_efield_on_grid(gse_context_t* ctx, double box_x, double box_y,
                                      double box_z, const void* phi, void* ex, void* ey,
                                      void* ez);

/* CpuGaussCharge<AT,CT>::calcDipoleSum (CpuGaussCharge.cpp:188-226):
 * dip[d] = sum_p (double)((rho_p hx hy hz) * h_d i_d) for d = x, y, z; each
 * term as the reference forms it in CT, the terms added in double in a fixed
 * order (not the reference's loop order).  rho is a CT grid (host or device),
 * dip three doubles (host or device). */
gse_status_t gse_gauss_dipole_sum(gse_context_t* ctx, double box_x, double box_y, double box_z,
                                  const void* rho, double* dip);

/* ---- virial (no reference counterpart) ----------------------------------- */

/* Reciprocal-space virial of the context's current rhoS (after gse_forward or
 * gse_spread_charge), in the energy's units: with E_k the mesh energy's
 * k-space terms (their sum is the energy of gse_calculate_energy),
 *   W_ab = sum_k E_k (delta_ab - 2 k_a k_b (1/k^2 + sigma^2/2)),
 * sigma the total Gaussian width (sigma^2 = 2 sigma1^2 + sigma2^2), the strain
 * derivative W_ab = -dE/d(eps_ab) of the Gaussian-split reciprocal energy.
 * virial receives xx, yy, zz, xy, xz, yz (6 doubles, host or device).  The
 * terms and their FP64 sum are formed on the GPU (r2c of rhoS, then one
 * reduction, deterministic); the context's k-space buffer is overwritten. */
gse_status_t gse_virial(gse_context_t* ctx, double* virial);

/* ---- reverse mode (no reference counterpart) ---------------------------- */

/* Vector-Jacobian product of one force evaluation (gse_forward) for the
 * scalar L with dL/dE = dLdE and dL/dF_i = (gfx[i], gfy[i], gfz[i]):
 * writes dq[i] = dL/dq_i and (dx, dy, dz)[i] = dL/dx_i.  The force-gradient
 * arrays may all be NULL (energy only).  The charge density and potential
 * grids are recomputed from xyzq (nothing is kept from an earlier forward
 * call); the adjoint source is spread with the gather's spherical cut,
 * solved with the same Green's function and gathered together with the
 * potential.  With dLdE = 1 and no force gradients, dq[i] is the potential
 * at atom i (dE/dq) and -(dx, dy, dz)[i] the cube-spread force. */
gse_status_t gse_adjoint(gse_context_t* ctx, int n, const void* xyzq, double dLdE,
                         const double* gfx, const double* gfy, const double* gfz, double* dq,
                         double* dx, double* dy, double* dz);

/* ---- Ewald reference sum --------------------------------------------------- */

/* CpuEwaldRecip::calcForceEnergy (CpuEwaldRecip.cpp:87-147) on the GPU in FP64:
 * E = sum over integer k != 0 with |k|^2 <= kcut^2 of
 * (2 pi / V) ccelec exp(-sigma^2 |k|^2 / 2) / |k|^2 |S(k)|^2 and the forces
 * -dE/dr (force arrays may all be NULL).  Independent of any context; it
 * allocates its own scratch and returns after the results are written.
 * kcut must lie in [1, 255]. */
gse_status_t gse_ewald_recip(int device, void* stream, double sigma, int kcut, double box_x,
                             double box_y, double box_z, double ccelec, int n, const double* xyzq,
                             double* energy, double* fx, double* fy, double* fz);

/* CpuEwaldDirect (CpuEwaldDirect.h:10-44): the constructor's sigma, rcut, box
 * and ccelec, setupExclusions (CpuEwaldDirect.cpp:31-40) and calcForceEnergy
 * (CpuEwaldDirect.cpp:45-131) in one call, on the GPU in FP64.  Over the pairs
 * at minimum-image distance r < rcut that are not excluded,
 * E = sum ccelec q_i q_j erfc(r / (sqrt(2) sigma)) / r
 *     - ccelec / sqrt(2 pi sigma^2) sum_i q_i^2,
 * and fx, fy, fz receive the gradient dE/dx of every atom, as the reference's
 * force arrays do (all three may be NULL).  Exclusions in CHARMM's format:
 * n_iblo14 = 0 for none (iblo14, inb14 may then be NULL), else n_iblo14 = n,
 * iblo14[a] the cumulative end of atom a's entries in inb14 (non-decreasing
 * from 0) and |inb14[k]| the 1-based partner; the pair (a, b), a < b, is
 * skipped when b is listed under a.  Exclusion arrays and energy are host
 * memory; xyzq (double4 per atom) and the force arrays host or device memory.
 * Independent of any context; it allocates its own scratch and returns after
 * the results are written.  The result does not depend on the order in which
 * the GPU runs its blocks. */
gse_status_t gse_ewald_direct(int device, void* stream, double sigma, double rcut, double box_x,
                              double box_y, double box_z, double ccelec, int n, const double* xyzq,
                              int n_iblo14, const int* iblo14, const int* inb14, double* energy,
                              double* fx, double* fy, double* fz);

/* ---- instrumentation (no reference counterpart) ------------------------ */

typedef enum gse_stage {
  GSE_STAGE_BIN = 0,          /* cell binning of atoms before the gather */
  GSE_STAGE_SPREAD = 1,       /* charge spreading (incl. grid clear/convert) */
  GSE_STAGE_FFT_FORWARD = 2,  /* r2c transform */
  GSE_STAGE_GREEN = 3,        /* Green's function multiply + k-space energy */
  GSE_STAGE_FFT_BACKWARD = 4, /* c2r transform */
  GSE_STAGE_GATHER = 5,       /* force gather */
  GSE_NUM_STAGES = 6
} gse_stage_t;

/* Record CUDA events around every stage on the context stream. */
gse_status_t gse_set_timing(gse_context_t* ctx, int enable);

/* Accumulated device milliseconds and launch counts per stage
 * (arrays of GSE_NUM_STAGES; either may be NULL); reset != 0 zeroes them. */
gse_status_t gse_get_timing(gse_context_t* ctx, double* ms_total, long long* counts, int reset);

/* The FP32 fused multiply-add rate this GPU sustains now, in TFLOP/s (2 flops
 * per fma), from a few ms of independent fmas on every SM: *tflops for the
 * scalar instruction, *tflops_packed (may be NULL) for the packed two-lane
 * form.  The spread and gather are bound by FP32 arithmetic and instruction
 * issue rather than by HBM; this is the denominator of their roofline.
 * Synchronises `stream` (a cudaStream_t on `device`). */
gse_status_t gse_measure_fp32_rate(int device, void* stream, double* tflops,
                                   double* tflops_packed);

/* Number of this library's own CUDA kernels the context has launched
 * (library calls such as cuFFT's are not counted). */
gse_status_t gse_get_launch_count(gse_context_t* ctx, long long* launches);

/* Which implementation paths the context takes (bits of *flags):
 *  GSE_PATH_TILED        brick-tiled spread and gather (grids >= 10 points per
 *                        side, stencil widths 9-15); otherwise atom-parallel kernels
 *  GSE_PATH_GREEN_IN_FFT the Green's-function multiply runs inside the c2r
 *                        transform as a cuFFT load callback, linked on the
 *                        context's first solve (grids of 64^3 points or more,
 *                        when the process's cuFFT and nvJitLink accept the
 *                        callback code -- not when an older cuFFT, such as the
 *                        one bundled with PyTorch, was loaded first); the energy
 *                        is then 1/2 ccelec h^3 sum rho phi in real space.
 *                        Otherwise a separate multiply kernel that also sums
 *                        the energy in k-space
 *  GSE_PATH_GRAPH        repeated gse_forward calls replay a captured CUDA graph
 *  GSE_PATH_OWN_FFT      mixed form on a cubic grid of M = 16 N2 points per side
 *                        (N2 = 4..12, e.g. 64, 80, 96, 128, 144, 192): the
 *                        context's own solve is this library's 3-D FFT, with
 *                        the int64 -> float conversion, the Green's multiply
 *                        and the k-space energy inside its passes, instead of
 *                        cuFFT (set GSE_B200_OWN_FFT=0 in the environment
 *                        before creating the context to keep cuFFT) */
#define GSE_PATH_TILED 1
#define GSE_PATH_GREEN_IN_FFT 2
#define GSE_PATH_GRAPH 4
#define GSE_PATH_OWN_FFT 8
gse_status_t gse_get_paths(gse_context_t* ctx, int* flags);

/* ---- spreading without allocation ------------------------------------- */

/* Largest grid (size_x*size_y*size_z points) gse_spread_mixed_noalloc takes. */
#define GSE_NOALLOC_MAX_GRID_POINTS 1048576

/* Mixed-precision charge spreading (the computation of gse_gauss_spread on a
 * GSE_PRECISION_MIXED context) that allocates no memory.  No counterpart in
 * the reference: it exists for callers that may not allocate device memory
 * while they run, e.g. a host engine whose own memory pool must remain the
 * only owner of device memory, or a time-step loop that cannot take the
 * synchronisation of cudaMalloc/cudaFree.
 *
 *  - xyzq (n float4 records, 16-byte aligned) and rho_out
 *    (size_x*size_y*size_z floats) must be device memory of the current
 *    device; the call is asynchronous on `stream` (a cudaStream_t, NULL =
 *    legacy default stream).
 *  - The int64 accumulation grid lives in a fixed device array of
 *    GSE_NOALLOC_MAX_GRID_POINTS values (8 MiB) that every GPU loading the
 *    library holds until the process exits; larger grids are rejected with
 *    GSE_ERR_INVALID_ARG.
 *  - The first call on a device looks up that array's device address, and
 *    again the first call in each further CUDA context on it (a caller that
 *    drives its own driver-API contexts has one copy of the array per
 *    context); make the first call on each device (and context) before any
 *    stream capture begins.  A cudaDeviceReset invalidates the address the
 *    library keeps: do not call this entry point after resetting a device
 *    that it has already run on.
 *  - All calls on a device share the one array and each call clears it
 *    first, so calls whose work overlaps on the GPU (different streams, no
 *    ordering between them) race and corrupt each other's results. */
gse_status_t gse_spread_mixed_noalloc(int size_x, int size_y, int size_z, double sigma,
                                      double rcut, int n, const float* xyzq, double box_x,
                                      double box_y, double box_z, float* rho_out, void* stream);

/* ---- many independent systems in one pass ------------------------------ */

/* No counterpart in the reference, which evaluates one system per object
 * (CpuGSEk<AT,CT>::calc_energy_force, CpuGSEk.h).  A batch holds S systems
 * that share sigma, kappa, lambda_sigma1 and ccelec (from the common
 * gse_params_t) but each have their own grid, box and atom count.  The mixed
 * form only (GSE_PRECISION_MIXED): positions are float {x,y,z,q}, results
 * double.  Every system computes exactly what a mixed gse_forward on its own
 * context computes, to float-rounding differences of the accumulation order
 * (grid values are summed in 64-bit fixed point, so a batch's own results do
 * not change from run to run). */
typedef struct gse_system {
  int size_x, size_y, size_z; /* grid points per side, each >= 10 */
  double box_x, box_y, box_z; /* orthorhombic box lengths */
  int n;                      /* atoms of this system (>= 0) */
} gse_system_t;

typedef struct gse_batch gse_batch_t;

/* Sizes and device buffers of a batch.  Atoms are numbered system after
 * system: system s owns atoms first_s .. first_s + n_s - 1, first_s the sum
 * of the earlier systems' n.  The device buffers stay valid until
 * gse_batch_destroy and are the ones a captured graph reads and writes. */
typedef struct gse_batch_info {
  int n_total, n_systems, n_size_classes;
  long long grid_points;           /* real grid points over all systems */
  int scatter_items, gather_items; /* (system, brick) work items */
  int scatter_ctas, gather_ctas;   /* persistent CTAs (autotuned) */
  int largest_first;               /* work items ordered by system size */
  void* xyzq;                      /* float4 [n_total] positions and charges */
  double* energies;                /* [n_systems] */
  double* forces;                  /* [3][n_total]: fx, then fy, then fz */
  double* dLdE;                    /* [n_systems] reverse-pass input */
  double* grad_forces;             /* [3][n_total] reverse-pass input */
  double* grad_out;                /* [4][n_total]: dL/dq, dL/dx, dL/dy, dL/dz */
  int fused;        /* 1: each direction is one persistent cooperative launch (every grid
                       side a multiple of 8 and at most 64); 0: one launch per stage */
  int gather_lanes; /* lanes per atom in the gather (autotuned on the fused path: 16 or 8) */
  int fused_ctas;   /* persistent CTAs of the fused launches */
  int graph_kernels; /* kernel nodes of the graph gse_batch_capture recorded (0: none) */
  int fused_available; /* 1: the fused schedule can run on this batch */
} gse_batch_info_t;

/* Build a batch: bins, grids grouped by size for strided FFT plans, and the
 * Green's-function table of every system (built in FP64). */
gse_status_t gse_batch_create(const gse_params_t* common, int n_systems,
                              const gse_system_t* systems, gse_batch_t** batch);
gse_status_t gse_batch_destroy(gse_batch_t* batch);
gse_status_t gse_batch_set_stream(gse_batch_t* batch, void* stream);
gse_status_t gse_batch_info(gse_batch_t* batch, gse_batch_info_t* info);

/* One evaluation of every system.  xyzq: n_total float4 records (host or
 * device; NULL = use the batch's xyzq buffer as it is).  energies [n_systems],
 * fx/fy/fz [n_total] may be host, device or NULL. */
gse_status_t gse_batch_forward(gse_batch_t* batch, const void* xyzq, double* energies,
                               double* fx, double* fy, double* fz);

/* Forward pass, then the reverse pass of L(E, F): dLdE [n_systems] and the
 * force cotangents gfx/gfy/gfz [n_total] (all three or none; NULL = zero) give
 * dL/dq, dL/dx, dL/dy, dL/dz [n_total] (each may be NULL). */
gse_status_t gse_batch_adjoint(gse_batch_t* batch, const void* xyzq, const double* dLdE,
                               const double* gfx, const double* gfy, const double* gfz,
                               double* dq, double* dx, double* dy, double* dz);

/* Capture one forward pass (and, if with_adjoint, the reverse pass) on the
 * batch's buffers into a CUDA graph; gse_batch_launch replays it on the
 * batch's stream, asynchronously.  Write inputs into the gse_batch_info
 * buffers and read results from them.  Changing the stream or re-tuning
 * drops the graph. */
gse_status_t gse_batch_capture(gse_batch_t* batch, int with_adjoint);
gse_status_t gse_batch_launch(gse_batch_t* batch);

/* Choose the launch schedule of the batch.  fused != 0: each direction as one
 * persistent cooperative kernel (binning, spread, the small-grid FFT solve with
 * the Green's multiply and energy, gather; or adjoint source, solve, reverse
 * gather, separated by grid-wide barriers), with gather_lanes (8 or 16) lanes
 * per atom in the gathers; only where every grid side is a multiple of 8 and
 * at most 64 (GSE_ERR_UNSUPPORTED otherwise).  fused == 0: one launch per
 * stage, persistent spread and gather kernels of scatter_ctas / gather_ctas
 * CTAs and cuFFT transforms per grid-size class.  largest_first orders the
 * work items by system size.  Drops a captured graph. */
gse_status_t gse_batch_set_schedule(gse_batch_t* batch, int fused, int gather_lanes,
                                    int largest_first, int scatter_ctas, int gather_ctas);

/* Time the launch schedules on the batch's current positions, each on a
 * forward and a reverse pass, and keep the fastest: the per-stage launches
 * (work-item order x persistent-CTA counts of spread and gather) and, where
 * the batch allows it, the fused launches (work-item order x lanes per atom of
 * the gathers: 16, two atoms per warp, or 8, four).  With
 * cache_path, the choice is appended to that text file under a key made of
 * the system count, grid-size histogram, atom count and SM count; with
 * use_cache != 0 a cached choice for the same key is taken without timing. */
gse_status_t gse_batch_autotune(gse_batch_t* batch, const char* cache_path, int use_cache);

#ifdef __cplusplus
}
#endif
#endif /* GSE_B200_H */
