/*
 * wp_api.h -- C ABI of the B200 (sm_100a) WaveletPotentials projection-and-recovery path.
 *
 * Every entry point takes plain pointers and sizes.  Field pointers are DEVICE pointers in the
 * reference layout (Utils.h:46-47: y fastest, element (x,y,z) of extents (DX,DY,DZ) at
 * y + x*DY + z*DX*DY) and MAC shapes (TestLocalProjection.cpp:536-542):
 *   xv (nx+1,ny,nz)  yv (nx,ny+1,nz)  zv (nx,ny,nz+1)  cells (nx,ny,nz)
 *   qx (nx,ny+1,nz+1) qy (nx+1,ny,nz+1) qz (nx+1,ny+1,nz); 2D: xv (nx+1,ny) yv (nx,ny+1) qz (nx+1,ny+1)
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).  Calls are
 * asynchronous on that stream unless they return a host scalar.  Errors come back as wp_status;
 * nothing calls exit().  wp_last_error() gives the message of the last failure on this thread.
 * Handles are independent: one handle per stream/thread.  Process-wide state is limited to caches
 * filled once (per-device SM counts, kernel attributes, the autotuner's choices per device and grid
 * extents, the launch counters and profiler records) and the static scratch of
 * wp_dst3d_solve_noalloc, whose sharing rules are stated at its declaration.
 *
 * The reference exposes no C ABI (cuWHHD_Export.h only defines an empty CUWHHD_API macro); each
 * declaration below names the reference C++ entry point it replaces.
 */
#ifndef WP_API_H
#define WP_API_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define CUWHHD_API __declspec(dllexport)
#else
#define CUWHHD_API __attribute__((visibility("default")))
#endif

typedef enum wp_status {
    WP_OK = 0,
    WP_ERR_INVALID_ARG = 1,   /* bad shape, null pointer, unknown enum */
    WP_ERR_UNSUPPORTED = 2,   /* valid request outside the implemented path (e.g. domain bc 'd') */
    WP_ERR_CUDA = 3,          /* a CUDA runtime call or launch failed */
    WP_ERR_WORKSPACE = 4,     /* caller workspace too small */
    WP_ERR_NOT_CONVERGED = 5, /* solve hit its cycle cap before the tolerance */
    WP_ERR_NONFINITE = 6,     /* NaN/Inf met in the input or residual */
    WP_ERR_DEVICE_WAIT = 7    /* a bounded wait inside a kernel gave up; that call's outputs are invalid,
                                 the handle stays usable */
} wp_status;

/* wavelet ids: same numeric values as the reference enum WaveletType (WaveletTypes.h:7-27) */
#define WP_CDF3_5 2  /* same lifting structure as CDF3.7, 5-tap second update (wp_dwt1d only) */
#define WP_CDF2_6 5  /* predict + 6-tap update, lines of 2^L + 1 (wp_dwt1d only) */
#define WP_CDF4_4 6  /* CDF4.6's structure with a 4-tap second update, lines of 2^L + 1 (wp_dwt1d only) */
#define WP_CDF4_6 7
#define WP_CDF2_8 10 /* predict + 8-tap update, lines of 2^L + 1 (wp_dwt1d only) */
#define WP_CDF3_7 11
#define WP_CDF2_0 16 /* CDF2.x's predict alone, lines of 2^L + 1, bc 'n' / 'd' (wp_dwt1d only) */
#define WP_CDF1_1 17 /* Haar, lines of 2^L, bc 'n' / 'd' (wp_dwt1d only) */
#define WP_CDF1_7 18 /* Haar predict + 7-tap update, lines of 2^L, bc 'n' / 'd' (wp_dwt1d only) */

/* precision modes of the multigrid solve */
#define WP_PREC_FP32 0  /* FP32 V-cycles, FP32 iterate; residual norms accumulated in FP64 */
#define WP_PREC_MIXED 1 /* FP32 V-cycles inside FP64 iterative refinement (FP64 defect + iterate) */
#define WP_PREC_FP64 2  /* FP64 V-cycles throughout (the reference's default DTYPE) */

CUWHHD_API const char* wp_last_error(void);
CUWHHD_API int wp_version(void);

/* Test-only: arms one withheld arrival for the next launch at `site`, so that one wait in it runs
   out after limit_seconds (in [1e-6, 2]) and the call returns WP_ERR_DEVICE_WAIT.  One shot.
   WP_WAIT_SITE_GRID_BARRIER: the last CTA of the persistent below-finest multigrid cycle skips the
   first grid barrier.  WP_WAIT_SITE_CONV_PIPELINE: the first CTA of the next tensor-core convolution
   (forward or weight gradient) does not load pipeline step `at`.  WP_WAIT_SITE_BATCH_PUBLISH: the
   next wp_batch_run of a WP_BATCH_PERSISTENT batch does not publish the phase that follows phase `at`
   of its first grid, so the persistent kernel's CTAs wait for work until the limit.  site 0 disarms.  Every other wait
   of that launch keeps its own limit; the kernels still wait for their copies in flight and free
   their tensor memory before they return.  No reference counterpart. */
#define WP_WAIT_SITE_GRID_BARRIER 1
#define WP_WAIT_SITE_CONV_PIPELINE 2
#define WP_WAIT_SITE_BATCH_PUBLISH 3
CUWHHD_API wp_status wp_debug_withhold_wait(int site, int at, double limit_seconds);

/* Instrumentation (no reference counterpart): number of kernels this library has launched since
   the last reset, and optional per-kernel-class timing with CUDA events on the launching stream.
   wp_profile_collect() synchronizes the device and returns the number of kernel classes;
   wp_profile_entry() reads one (name, launches, total ms, algorithmic bytes moved). */
CUWHHD_API void wp_profile_enable(int on);
CUWHHD_API void wp_profile_reset(void);
CUWHHD_API long long wp_launch_count(void);
CUWHHD_API int wp_profile_collect(void);
CUWHHD_API int wp_profile_entry(int i, char* name, int name_cap, long long* launches, double* ms, double* bytes);

/* ------------------------------------------------------------------ 1D transforms ------- */
/* Full-depth multilevel 1D lifting transform (CDF3.7 / CDF4.6 and the other families the reference
   registers: CDF3.5, CDF4.4, CDF2.6, CDF2.8; bc 'n' | 'd' | 'z') along
   direction 'x' | 'y' | 'z' of a (dim_x, dim_y, dim_z) array; dst may equal src.
   Replaces CuWHHDForward::Solve1D(dst, src, int3 dim, level, direction, bc, type, is_forward)
   (cuWHHDForward.cuh:20-23, cuWHHDForward.cu:1122-1153). */
CUWHHD_API wp_status wp_dwt1d(float* dst, const float* src, int dim_x, int dim_y, int dim_z, int levels,
                              char direction, char bc, int wavelet, int forward, void* stream);
CUWHHD_API wp_status wp_dwt1d_f64(double* dst, const double* src, int dim_x, int dim_y, int dim_z, int levels,
                                  char direction, char bc, int wavelet, int forward, void* stream);

/* Diagonal band of the inner-product table ||B_i||^2 of the synthesis basis, computed on the GPU
   in FP64 and copied to host `out[dim]` (synchronous).  Replaces CuGetInnerProduct::GenerateIp
   (cuGetInnerProduct.cu:92-126; only band 0 is read by the projection kernels). */
CUWHHD_API wp_status wp_ip_diag(double* out, int dim, int wavelet, char bc);

/* ---------------------------------------------------------- potential recovery 3D ------- */
typedef struct wp_recover3d wp_recover3d;
/* Replaces CuWaveletPotentialRecover3D(int3 dim, DTYPE3 dx, char bc, WaveletType curl,
   WaveletType div) (cuWaveletPotentialRecover3D.cuh:11-12, .cu:6-12).  nx,ny,nz powers of two
   >= 4; bc 'n' (zero-normal-flux walls) or 'd' (Dirichlet walls: the curl wavelet takes bc 'd', the
   div wavelet 'n', and the projection is cuProjectLocal_q_3d_nq_ccc, cuDivLocalProject3D.cu:4474-4877;
   such a handle recovers fields with nonzero wall flux).  Allocates its own temporaries on the
   current device. */
CUWHHD_API wp_status wp_recover3d_create(wp_recover3d** h, int nx, int ny, int nz, double dx, double dy, double dz,
                                         char bc, int curl_wavelet, int div_wavelet);
/* Replaces CuWaveletPotentialRecover3D::Solve(qx,qy,qz,xv,yv,zv) (cuWaveletPotentialRecover3D.cu:16-61):
   forward analysis, local projection, inverse synthesis.  xv..zv are read only. */
CUWHHD_API wp_status wp_recover3d_run(wp_recover3d* h, float* qx, float* qy, float* qz, const float* xv,
                                      const float* yv, const float* zv, void* stream);
/* Replaces CuDivLocalProject3D::ProjectLocal_q_ccc(qx,qy,qz,xv_lwt,yv_lwt,zv_lwt,levels)
   (cuDivLocalProject3D.cu:5273-5308): coefficient-space projection only. */
CUWHHD_API wp_status wp_recover3d_project(wp_recover3d* h, float* qx, float* qy, float* qz, const float* xv_lwt,
                                          const float* yv_lwt, const float* zv_lwt, void* stream);
/* Replaces CuWaveletPotentialRecover3D::CutCoefficients(qx_out, qy_out, qz_out, qx, qy, qz, level)
   (cuWaveletPotentialRecover3D.cu:123-239): analyses the potential with the recovery's synthesis
   wavelets, clears the coefficients of every index whose level along some axis is below `level`
   (with the reference's coupling of the three components), and synthesises the result into the
   _out arrays (which may alias the inputs).  level in [0, min(log2 n)]: 0 returns the potential.
   Handles with bc 'n' only (WP_ERR_UNSUPPORTED otherwise). */
CUWHHD_API wp_status wp_recover3d_cut(wp_recover3d* h, float* qx_out, float* qy_out, float* qz_out, const float* qx,
                                      const float* qy, const float* qz, int level, void* stream);
CUWHHD_API wp_status wp_recover3d_destroy(wp_recover3d* h);

/* ---------------------------------------------------------- potential recovery 2D ------- */
typedef struct wp_recover2d wp_recover2d;
/* Replaces CuWaveletPotentialRecover2D(int2 dim, DTYPE2 dx, char bc, curl, div)
   (cuWaveletPotentialRecover2D.cuh:11-12).  bc 'n' (zero-normal-flux walls: cuProjectLocal_q_single)
   or 'd' (Dirichlet walls: the div wavelet takes 'n' and the projection is cuProjectLocal_q_single_n,
   cuDivLocalProject.cu:1047-1460). */
CUWHHD_API wp_status wp_recover2d_create(wp_recover2d** h, int nx, int ny, double dx, double dy, char bc,
                                         int curl_wavelet, int div_wavelet);
/* Replaces CuWaveletPotentialRecover2D::Solve(qz, xv, yv) (cuWaveletPotentialRecover2D.cu:16-36). */
CUWHHD_API wp_status wp_recover2d_run(wp_recover2d* h, float* qz, const float* xv, const float* yv, void* stream);
/* Replaces CuDivLocalProject::ProjectSingle(qz, xv_lwt, yv_lwt) (cuDivLocalProject.cu:2162-2198). */
CUWHHD_API wp_status wp_recover2d_project(wp_recover2d* h, float* qz, const float* xv_lwt, const float* yv_lwt,
                                          void* stream);
CUWHHD_API wp_status wp_recover2d_destroy(wp_recover2d* h);

/* ---------------------------------------------------- fractional multigrid 3D / 2D ------- */
/* coarse-to-fine transfer of the V-cycle */
#define WP_PROLONG_CONSTANT 0  /* the reference's piecewise-constant prolongation (cuProlongate3D.cu:594-617) */
#define WP_PROLONG_TRILINEAR 1 /* cell-centred trilinear: h-independent convergence for V(2,2), omega 2/3 */
/* first iterate of the tolerance-driven solve: zero, or a full-multigrid start (the right-hand side
   restricted to every level, the coarsest solved, then prolongation + one V-cycle per finer level),
   which costs about two V-cycles of work and counts as one cycle in the report */
#define WP_START_ZERO 0
#define WP_START_FMG 1

typedef struct wp_mg_params {
    int max_cycles;   /* cap on V-cycles (or refinement steps) */
    int nu1, nu2;     /* pre / post weighted-Jacobi sweeps */
    double omega;     /* Jacobi weight (reference default 0.8, cuMultigridFrac3D.cuh:17) */
    double rel_tol;   /* stop when ||f - A p|| / ||f|| <= rel_tol; <= 0 runs exactly max_cycles */
    int precision;    /* WP_PREC_FP32 | WP_PREC_MIXED | WP_PREC_FP64 */
    int prolongation; /* WP_PROLONG_CONSTANT | WP_PROLONG_TRILINEAR */
    int start;        /* WP_START_ZERO | WP_START_FMG (ignored when an initial iterate is given) */
    int host_loop;    /* 0: WP_PREC_MIXED tolerance solves run their cycle loop on the device (a CUDA
                         graph whose while-node repeats cycle + defect + convergence test, no host
                         round trip per cycle); 1: the host tests convergence after every cycle.
                         Both give the same iterates, cycle counts and residual history. */
    int inner_cycles; /* WP_PREC_MIXED: FP32 V-cycles per refinement step (0 or 1: one; 2: the
                         FP32 correction equation is solved with two cycles before the FP64 update
                         and defect, which halves the FP64 defect passes; the tolerance is then
                         tested every inner_cycles cycles and history[] holds one entry per step) */
} wp_mg_params;

typedef struct wp_mg_report {
    int cycles;             /* V-cycles executed */
    double rel_residual;    /* final ||f - A p|| / ||f|| (FP64) */
    double history[64];     /* relative residual after each refinement step (each V-cycle outside
                               WP_PREC_MIXED with inner_cycles > 1); first min(steps,64) */
    int steps;              /* entries of history written (= cycles unless inner_cycles > 1) */
} wp_mg_report;

typedef struct wp_mgfrac3d wp_mgfrac3d;
/* Replaces CuMultigridFrac3D(Ax, Ay, Az, int3 dim, DTYPE3 dx, char bc) (cuMultigridFrac3D.cuh:15,
   .cu:9-134): copies the face fractions and builds the coarse hierarchy (ceil halving until the
   smallest extent is 1).  bc 'n' only. */
CUWHHD_API wp_status wp_mgfrac3d_create(wp_mgfrac3d** h, const float* ax, const float* ay, const float* az, int nx,
                                        int ny, int nz, double dx, double dy, double dz, char bc, void* stream);
/* Replaces CuMultigridFrac3D::Solve(dst, pre_v, f, n_iters, nu1, nu2, weight) (cuMultigridFrac3D.cu:249-265):
   exactly n_iters V-cycles in FP32.  pre_v may be NULL (zero start) or equal dst. */
CUWHHD_API wp_status wp_mgfrac3d_solve(wp_mgfrac3d* h, float* dst, const float* pre_v, const float* f, int n_iters,
                                       int nu1, int nu2, double weight, void* stream);
/* Replaces CuMultigridFrac3D::Solve_index(dst, pre_v, f, n_iters, nu1, nu2, weight)
   (cuMultigridFrac3D.cu:347-420, index lists InitIndex :189-229, CuBoundSelector::SelectByFrac
   cuBoundSelector.cu:4-32): n_iters FP32 V-cycles that sweep, restrict and prolong only the cells
   with a face fraction >= 1e-12 ("listed" cells), for mostly-solid domains.  As the reference:
   post-smoothing runs nu1 sweeps (nu2 is checked and otherwise unused); unlisted finest cells keep
   their start value (pre_v, or 0); the cycle descends while the next level lists a cell, then runs
   the coarsest solve; the residual workspace is shared by all levels and kept by the handle between
   calls (zero when the lists are built), and the restriction reads it at every child of a listed
   coarse cell.  The first call builds the lists (synchronous); 3D handles only. */
CUWHHD_API wp_status wp_mgfrac3d_solve_index(wp_mgfrac3d* h, float* dst, const float* pre_v, const float* f,
                                             int n_iters, int nu1, int nu2, double weight, void* stream);
/* The same cycle in FP64, the reference's default DTYPE (DoubleUseDefine.h): dst, pre_v and f are
   double arrays of cells; it has its own residual workspace.  It overwrites the level arrays that
   hold the FP64 tolerance solve's iterate (wp_mgfrac3d_iterate64 then reports none). */
CUWHHD_API wp_status wp_mgfrac3d_solve_index64(wp_mgfrac3d* h, double* dst, const double* pre_v, const double* f,
                                               int n_iters, int nu1, int nu2, double weight, void* stream);
/* Listed cells (the reference's v_index_size_) and 32-cell row segments per level, first
   min(cap, levels); builds the lists if needed.  No reference counterpart. */
CUWHHD_API wp_status wp_mgfrac3d_index_sizes(wp_mgfrac3d* h, long long* cells, long long* segments, int cap,
                                             int* levels, void* stream);
/* Tolerance-driven solve with a precision mode; synchronous (reads residual norms on the host).
   Solves the compatible problem A p = f - m, m = mean of f over the active cells (diag > 0), so the
   FP32 rounding of f does not floor the residual; the residual reported is ||f - m - A p|| / ||f||.
   Returns WP_ERR_NOT_CONVERGED (dst still holds the last iterate) when max_cycles is reached. */
CUWHHD_API wp_status wp_mgfrac3d_solve_tol(wp_mgfrac3d* h, float* dst, const float* pre_v, const float* f,
                                           const wp_mg_params* params, wp_mg_report* report, void* stream);
/* Replaces CuMultigridFrac3D::GetResdualError(dst, f) (cuMultigridFrac3D.cu:329-333): returns
   ||f - A v||_2 / ||f||_2 with FP64 accumulation (synchronous). */
CUWHHD_API wp_status wp_mgfrac3d_residual(wp_mgfrac3d* h, const float* v, const float* f, double* rel_residual,
                                          void* stream);
/* Copies the FP64 iterate of the last WP_PREC_MIXED / WP_PREC_FP64 solve into dst (device, cells);
   WP_ERR_INVALID_ARG if the handle has not run such a solve.  No reference counterpart (the
   reference iterate is DTYPE). */
CUWHHD_API wp_status wp_mgfrac3d_iterate64(wp_mgfrac3d* h, double* dst, void* stream);
/* The device address of that FP64 iterate inside the handle (no copy; valid until the handle's
   next solve or its destruction); WP_ERR_INVALID_ARG if the handle has not run such a solve.  No
   reference counterpart. */
CUWHHD_API wp_status wp_mgfrac3d_iterate64_view(wp_mgfrac3d* h, const double** out);
CUWHHD_API wp_status wp_mgfrac3d_destroy(wp_mgfrac3d* h);
/* Tile-shape autotuner (no reference counterpart): times the column-walking stencil kernels of
   every level (Jacobi sweep, fused residual-restriction, FP64 defect) over candidate z-chunks and
   keeps the fastest per level; results are independent of the choice.  Synchronous; overwrites
   the handle's work arrays (not the FP64 iterate).  Choices are cached per device and extents for
   the process.  Each candidate is timed as the median of single launches, after an L2 flush for
   levels larger than 16 MB, among chunks that give at least two CTAs per SM (when the level has
   that many columns).  wp_mgfrac3d_tiles reports 3 chunks per level (jacobi, restrict, defect),
   and where not NULL their kernel variants (see wp_mgfrac3d_set_tile) and tuned median time per
   sweep in ms (0 where not tuned). */
CUWHHD_API wp_status wp_mgfrac3d_autotune(wp_mgfrac3d* h, void* stream);
CUWHHD_API wp_status wp_mgfrac3d_tiles(const wp_mgfrac3d* h, int* zc, int* variant, float* ms, int cap,
                                       int* levels);
/* Pins one level's choice: kind 0 (Jacobi: variant 0-2 one sweep per launch with default / >= 3 /
   >= 4 CTAs per SM register budgets, 3 two sweeps per launch, 4 TMA-staged rows on persistent CTAs,
   5 the next planes' loads issued ahead with cp.async, 6 one cell per thread; 3-6 FP32 3D levels
   only), 1 (restriction: variant 0-2 the same register budgets, 3 pipelined, 4 one cell per
   thread) or 2 (FP64 defect: 0 quads, 1 pipelined); zc <= 0 restores the heuristic chunk.  Kind 3
   (level and zc ignored): the levels below the finest run as one persistent cooperative launch
   (variant 1, the default where the autotuner finds it faster) or launch by launch (variant 0). */
CUWHHD_API wp_status wp_mgfrac3d_set_tile(wp_mgfrac3d* h, int level, int kind, int zc, int variant);
/* Uniform rows of one level (no reference counterpart): the number of (x, z) rows of cells whose
   interior face fractions are all exactly 1, which the column kernels stream without reading any
   fraction, and the number of rows (nx nz); counted when the handle is built.  For traffic
   accounting. */
CUWHHD_API wp_status wp_mgfrac3d_uniform_rows(const wp_mgfrac3d* h, int level, long long* uniform, long long* rows);

typedef struct wp_mgfrac2d wp_mgfrac2d;
/* Replaces CuMultigridFrac2D(Ax, Ay, int2 dim, DTYPE2 dx, char bc) (cuMultigridFrac2D.cu:28-111). */
CUWHHD_API wp_status wp_mgfrac2d_create(wp_mgfrac2d** h, const float* ax, const float* ay, int nx, int ny, double dx,
                                        double dy, char bc, void* stream);
/* Replaces CuMultigridFrac2D::Solve (cuMultigridFrac2D.cu:151-166). */
CUWHHD_API wp_status wp_mgfrac2d_solve(wp_mgfrac2d* h, float* dst, const float* pre_v, const float* f, int n_iters,
                                       int nu1, int nu2, double weight, void* stream);
CUWHHD_API wp_status wp_mgfrac2d_solve_tol(wp_mgfrac2d* h, float* dst, const float* pre_v, const float* f,
                                           const wp_mg_params* params, wp_mg_report* report, void* stream);
/* Replaces CuWeightedJacobi::GetFracRhs(v, f, Ax, Ay, dim, dx, dy, dx_e, bc) (cuWeightedJacobi.cu:789-811). */
CUWHHD_API wp_status wp_mgfrac2d_residual(wp_mgfrac2d* h, const float* v, const float* f, double* rel_residual,
                                          void* stream);
CUWHHD_API wp_status wp_mgfrac2d_destroy(wp_mgfrac2d* h);

/* ------------------------------------------------------------- field operators ------- */
/* b = -div(a u) (CuConvergence::GetB_3d_frac_vel, cuConvergence.cu:427-447).  ax, ay, az all NULL
   means fully open faces (the divergence of an already fraction-weighted field). */
CUWHHD_API wp_status wp_divergence_frac3d(float* b, const float* xv, const float* yv, const float* zv, const float* ax,
                                          const float* ay, const float* az, int nx, int ny, int nz, double dx,
                                          double dy, double dz, void* stream);
/* 2D form (CuConvergence::GetB_2d_frac_vel); ax, ay both NULL means fully open faces. */
CUWHHD_API wp_status wp_divergence_frac2d(float* b, const float* xv, const float* yv, const float* ax, const float* ay,
                                          int nx, int ny, double dx, double dy, void* stream);
/* u <- (u - grad p) [* a]: CuGradient::Gradient3D_Frac_P (cuGradient.cu:2520-2540) followed by
   CudaMatAdd(-1) and CudaMatMul(a) (TestLocalProjection.cpp:672-680), fused. */
CUWHHD_API wp_status wp_grad_subtract_frac3d(float* xv, float* yv, float* zv, const float* p, const float* ax,
                                             const float* ay, const float* az, int nx, int ny, int nz, double dx,
                                             double dy, double dz, int multiply_frac, void* stream);
/* The same update with the FP64 pressure iterate of a WP_PREC_MIXED / WP_PREC_FP64 solve
   (wp_mgfrac3d_iterate64_view): the gradient and the difference are formed in FP64 and rounded
   once to the FP32 face value, as the reference's default FP64 build forms them (DoubleUseDefine.h:5,
   cuGradient.cu:1952-2000).  No reference counterpart as a separate entry point. */
CUWHHD_API wp_status wp_grad_subtract_frac3d_p64(float* xv, float* yv, float* zv, const double* p, const float* ax,
                                                 const float* ay, const float* az, int nx, int ny, int nz, double dx,
                                                 double dy, double dz, int multiply_frac, void* stream);
CUWHHD_API wp_status wp_grad_subtract_frac2d(float* xv, float* yv, const float* p, const float* ax, const float* ay,
                                             int nx, int ny, double dx, double dy, int multiply_frac, void* stream);
/* max |x| over n elements, FP64 result to host (CudaFindMaxValue, cudaMath.cu:1269-1280, without
   copying the array to the host).  Synchronous. */
CUWHHD_API wp_status wp_max_abs(const float* x, size_t n, double* out, void* stream);

/* Signed distance (positive in fluid) to a union of spheres at cell centres (cuInitLsSphere,
   cuSolidLevelSet3D.cu:11-27); centers/radii are HOST arrays (3*count, count). */
CUWHHD_API wp_status wp_sdf_spheres3d(float* sdf, int nx, int ny, int nz, double dx, const double* centers,
                                      const double* radii, int count, void* stream);
/* Union of axis-aligned boxes (HOST lo/hi arrays, 3*count each) into an existing level set (min);
   exact box signed distance.  No reference counterpart (the reference builds spheres only); used
   for the mixed-obstacle configurations. */
CUWHHD_API wp_status wp_sdf_boxes3d(float* sdf, int nx, int ny, int nz, double dx, const double* lo, const double* hi,
                                    int count, void* stream);
/* Face open fractions from a level set (cuGetAx/Ay/Az, cuSolidLevelSet3D.cu:36-90). */
CUWHHD_API wp_status wp_fractions3d(float* ax, float* ay, float* az, const float* sdf, int nx, int ny, int nz,
                                    double dx, void* stream);
/* Replaces the static CuSolidLevelSet3D::GetFrac(ax, ay, az, ls, dim, dx) (cuSolidLevelSet3D.cu:356-372,
   kernels cuGetAx/Ay/Az_divide :164-316): face open fractions of an arbitrary level set (positive in
   fluid): open where the quadratic interpolant at the face centre exceeds dx, closed at or below
   -dx, otherwise the share of 128 x 128 sub-face samples where the trilinear interpolant is
   positive.  FP64 arithmetic; ls FP32.  Extents >= 2 and fewer than 2^30 faces per axis. */
CUWHHD_API wp_status wp_fractions3d_subsampled(float* ax, float* ay, float* az, const float* ls, int nx, int ny,
                                               int nz, double dx, void* stream);
/* Replace CuFastSweeping::Solve(ls, dim, dx, n_iters) and ReinitLevelSet(ls, dim, dx, n_iters)
   (cuFastSweeping.cu:215-257, 383-396): n_iters eikonal updates of every cell above -1e-12 from its
   neighbours (upwind |grad d| = 1, spacing dx on every axis; cells at or below -1e-12 are the fixed
   sources); Reinit negates, sweeps, negates back and sweeps again, so both sides become distances.
   Each iteration reads the previous one (the reference updates in place from concurrent threads):
   one cell of propagation per iteration, the same fixed point. */
CUWHHD_API wp_status wp_fast_sweep_solve(float* ls, int nx, int ny, int nz, double dx, int n_iters, void* stream);
CUWHHD_API wp_status wp_fast_sweep_reinit(float* ls, int nx, int ny, int nz, double dx, int n_iters, void* stream);
/* Replaces CuFastSweeping::ParticlesToLs(ls, x, dim, n_pars, dx, radius, max_dis, n_iters)
   (cuFastSweeping.cu:259-349): a level set (negative inside) of balls of `radius` around `count`
   particles (xyz: device array of count x 3 floats, positions in the domain's units): rough
   distances at the 8 cells around each particle, then two sign flips each followed by n_iters
   eikonal sweeps (wp_fast_sweep_solve), then negation.  Cells outside the grid are skipped (the
   reference writes them). */
CUWHHD_API wp_status wp_particles_to_ls(float* ls, const float* xyz, int count, int nx, int ny, int nz, double dx,
                                        double radius, double max_dis, int n_iters, void* stream);
/* Replaces CuFastSweeping::ParticlesToLsNarrow(ls, x, dim, n_pars, dx, radius, max_dis, n_iters)
   (cuFastSweeping.cu:352-385): ls on entry is the start (a narrow band or a previous level set, not
   filled); the particles' rough distances lower it, then n_iters sweeps, negation, n_iters sweeps.
   max_dis is unused (as in the reference).  Cells outside the grid are skipped (the reference writes
   them). */
CUWHHD_API wp_status wp_particles_to_ls_narrow(float* ls, const float* xyz, int count, int nx, int ny, int nz,
                                               double dx, double radius, double max_dis, int n_iters, void* stream);
/* 2D: circle level set (CuSolidLevelSet2D, cuSolidLevelSet2D.cu) and face fractions. */
CUWHHD_API wp_status wp_sdf_circles2d(float* sdf, int nx, int ny, double dx, const double* centers, const double* radii,
                                      int count, void* stream);
CUWHHD_API wp_status wp_fractions2d(float* ax, float* ay, const float* sdf, int nx, int ny, double dx, void* stream);

/* ------------------------------------------------------------- DST-I Poisson ------- */
typedef struct wp_dst3d wp_dst3d;
/* Replaces CuDst3D(int3 dim, DTYPE3 dx) (cuDst3D.cu:202-255): Dirichlet Poisson solver by DST-I. */
CUWHHD_API wp_status wp_dst3d_create(wp_dst3d** h, int nx, int ny, int nz, double dx, double dy, double dz);
/* Replaces CuDst3D::Solve(dst, f) (cuDst3D.cu:265-341): FP64 device arrays of nx*ny*nz cells,
   dst may equal f; solves -lap_h p = f with p = 0 outside the grid (scaled by dx*dy as the reference). */
CUWHHD_API wp_status wp_dst3d_solve(wp_dst3d* h, double* dst, const double* f, void* stream);
CUWHHD_API wp_status wp_dst3d_destroy(wp_dst3d* h);

/* ------------------------------------------------- sweep + DST potential recovery ------- */
typedef struct wp_sweep3d wp_sweep3d;
/* Replaces CuParallelSweep3D(int3 dim, DTYPE3 dx, char bc) (cuParallelSweep3D.cu:868-887), the
   reference's comparison baseline for the wavelet recovery; bc 'n' or 'd' (others:
   WP_ERR_UNSUPPORTED).  A bc 'n' handle owns the DST-I solver of the (n-1)^3 interior nodes. */
CUWHHD_API wp_status wp_sweep3d_create(wp_sweep3d** h, int nx, int ny, int nz, double dx, double dy, double dz,
                                       char bc);
/* Replaces CuParallelSweep3D::Solve(qx, qy, qz, xv, yv, zv) (cuParallelSweep3D.cu:939-966): a vector
   potential with curl q = u for a divergence-free u with no normal flux: qx, qy integrate yv, -xv
   along z from 0 on z = 0, qz = 0 except the top plane, which takes the x-integral of qx's top
   plane (then cleared).  bc 'd' (SetQxQyBoundary, :925-937): qy's z = 0 plane is the x-integral of
   zv's bottom face, no top-plane step (zv is read only then).  q in the edge shapes of
   wp_recover3d_run. */
CUWHHD_API wp_status wp_sweep3d_solve(wp_sweep3d* h, float* qx, float* qy, float* qz, const float* xv,
                                      const float* yv, const float* zv, void* stream);
/* Replaces CuParallelSweep3D::SolveFromMid(qx, qy, qz, xv, yv, zv, int3 mid) (cuParallelSweep3D.cu:967-984):
   qz = 0, qx's plane mid_z = 0, qy's plane mid_z the x-integral of zv's plane mid_z both ways from 0
   at row mid_x (the reference leaves that row as the caller's buffer had it), then the z integrals of
   Solve both ways from plane mid_z.  mid_y is unused (as in the reference). */
CUWHHD_API wp_status wp_sweep3d_solve_from_mid(wp_sweep3d* h, float* qx, float* qy, float* qz, const float* xv,
                                               const float* yv, const float* zv, int mid_x, int mid_y, int mid_z,
                                               void* stream);
/* Replaces CuParallelSweep3D::Project(qx, qy, qz) with bc 'n' = ProjectZero
   (cuParallelSweep3D.cu:1043-1081, 1316-1326): q -= grad phi with -lap phi = -div q on the interior
   nodes (DST-I), phi = 0 on the walls, in place.  bc 'd' (ProjectD) returns WP_ERR_UNSUPPORTED: the
   reference's run of it at 16^3 raised an illegal address, so it is not built. */
CUWHHD_API wp_status wp_sweep3d_project(wp_sweep3d* h, float* qx, float* qy, float* qz, void* stream);
CUWHHD_API wp_status wp_sweep3d_destroy(wp_sweep3d* h);
/* Replaces CuParallelSweep3D(int2, DTYPE2, char)::Solve(qz, xv, yv) (cuParallelSweep3D.cu:986-998):
   qz ((nx+1) x (ny+1)) = 0 on x = 0 (bc 'n') or, with bc 'd', the y-integral of xv's x = 0 column
   there (from qz(0, 0) = 0, which the reference leaves as the caller's buffer had it), then the
   -x-integral of yv. */
CUWHHD_API wp_status wp_sweep2d_solve(float* qz, const float* xv, const float* yv, int nx, int ny, double dx,
                                      double dy, char bc, void* stream);

/* Allocation-free DST-I Poisson solve.  No reference counterpart (CuDst3D allocates its buffers in
   its constructor).  Same result as wp_dst3d_create + wp_dst3d_solve, but no handle and no device
   allocation on any call: the three DST-I matrices and the intermediate buffer live in one static
   device array of 3*64*64 + 64^3 doubles (2.2 MB) inside the library.  For callers that cannot
   allocate: a solver running under a fixed device-memory budget whose pool is already committed,
   or a stream-ordered loop next to other streams where cudaFree's implicit device synchronization
   would stall them.
   - Limits: every extent <= WP_DST_NOALLOC_MAX_EXTENT and nx*ny*nz <= WP_DST_NOALLOC_MAX_CELLS;
     larger grids return WP_ERR_INVALID_ARG (use wp_dst3d_create / wp_dst3d_solve).
   - Nothing in the scratch has to start at zero: every call writes each word it reads.
   - The first call on each device resolves the scratch address (cudaGetSymbolAddress, with that
     device current); make that first call an ordinary one, before any stream capture.  The address
     is kept for the rest of the process: after cudaDeviceReset on a device, do not call this entry
     point on that device again (the cached address belongs to the destroyed context).
   - The scratch is shared by all calls on a device: two calls that overlap in time (different
     streams, or different host threads without ordering) race on it and give wrong results.
     Order them (same stream, or events).
   dst and f are FP64 device arrays of nx*ny*nz cells in the INDEX3D layout; dst may equal f. */
#define WP_DST_NOALLOC_MAX_EXTENT 64
#define WP_DST_NOALLOC_MAX_CELLS (64 * 64 * 64)
CUWHHD_API wp_status wp_dst3d_solve_noalloc(double* dst, const double* f, int nx, int ny, int nz, double dx,
                                            double dy, double dz, void* stream);

/* ------------------------------------------------------------- tensor-core convolutions ------- */
/* No reference counterpart (the reference has no learned component): the 3x3x3 zero-padded
   convolutions of the warm-start network, on the tcgen05 tensor cores (BF16 operands, FP32
   accumulation).  Volumes are channels-last BF16 [z][x][y][c] with c in {16, 32, 64}; nx and ny are
   powers of two.  Weights of input part p are BF16 [27][cout][cin_p], tap = (dz*3 + dx)*3 + dy for
   the offsets (dz-1, dx-1, dy-1).
   wp_conv3_forward: out = relu?( conv(x0, w0) [+ conv(x1, w1)] + bias + addend ) and, when mask is
   given, zero where mask <= 0 (x1/w1, bias, addend, mask may be NULL; bias is FP32 [cout]; addend
   and mask are BF16 volumes of cout channels).  With the weights transposed and flipped
   ([26 - tap][cin][cout]) the same call is the input gradient.
   wp_conv3_wgrad: dw[27][cout][cin] += sum_v gy[v][co] x[v + off(tap)][ci] in FP32 (caller zeroes
   dw).  Both synchronize the stream to report a pipeline timeout. */
CUWHHD_API wp_status wp_conv3_forward(void* out, const void* x0, int cin0, const void* w0, const void* x1, int cin1,
                                      const void* w1, const float* bias, int cout, int nx, int ny, int nz, int relu,
                                      const void* addend, const void* mask, void* stream);
CUWHHD_API wp_status wp_conv3_wgrad(float* dw, const void* x, int cin, const void* gy, int cout, int nx, int ny,
                                    int nz, void* stream);

/* ------------------------------------------------------------- seeded generators ------- */
/* No reference counterpart.  Gaussian random fields with power spectrum |k|^slope as sums of random
   Fourier modes 0 < |k| <= kmax (kmax <= 32) over the unit domain, variance scaled to rms^2; modes
   are drawn on the host from std::mt19937_64(seed), so a seed gives the same field everywhere.
   wp_random_field3d samples one field at cell indices (x/nx, y/ny, z/nz) into out (nz, nx, ny).
   wp_velocity3d writes the MAC velocity u = curl(psi) + grad(phi) (psi: three edge fields with
   psi_slope/psi_rms, phi: a cell field with phi_slope/phi_rms), wall-normal faces zero. */
CUWHHD_API wp_status wp_random_field3d(float* out, int nx, int ny, int nz, double slope, double rms, int kmax,
                                       unsigned long long seed, void* stream);
CUWHHD_API wp_status wp_velocity3d(float* xv, float* yv, float* zv, int nx, int ny, int nz, unsigned long long seed,
                                   double psi_slope, double psi_rms, double phi_slope, double phi_rms, int kmax,
                                   void* stream);

/* ------------------------------------------------------------- warm-start network ------- */
/* No reference counterpart.  A 3-level 3D U-Net (3x3x3 convolutions 16/32/64 channels with ReLU,
   2x2x2 average pooling, nearest upsampling, concatenated skips, 1x1 head; BF16 weights and
   activations, FP32 accumulation on the tensor cores) that maps the multigrid right-hand side b
   and the solid level set sdf (FP32 cell arrays, INDEX3D layout) to a starting guess p for
   wp_mgfrac3d_solve_tol.  nx, ny: powers of two >= 16; nz a multiple of 4.  The multigrid then
   runs to the same tolerance, so the guess can only remove cycles (callers fall back to a zero
   start when the guess's residual exceeds ||b||).
   wp_unet_train_step: one Adam step (lr) on the loss mean over fluid cells (sdf > 0) of
   (p/rms(b) - p_target/rms(b) - mean error)^2; *loss (may be NULL) receives the loss before the
   step (synchronizes).  lr = 0 computes the gradients only.
   wp_unet_params: parameters (which = 0) or last gradients (which = 1) as one FP32 vector: per
   convolution its part weights [27][cout][cin_p] then bias, in the order c1a c1b c2a c2b c3a c3b
   d2a d2b d1a d1b, then the head's 16 weights and bias; host = NULL returns the count only. */
typedef struct wp_unet wp_unet;
CUWHHD_API wp_status wp_unet_create(wp_unet** h, int nx, int ny, int nz, unsigned long long seed);
CUWHHD_API wp_status wp_unet_predict(wp_unet* h, float* p, const float* b, const float* sdf, double h_cell,
                                     void* stream);
CUWHHD_API wp_status wp_unet_train_step(wp_unet* h, const float* b, const float* sdf, const float* p_target,
                                        double h_cell, double lr, double* loss, void* stream);
CUWHHD_API wp_status wp_unet_params(wp_unet* h, int which, float* host, size_t cap, size_t* count);
CUWHHD_API wp_status wp_unet_set_params(wp_unet* h, const float* host, size_t count);
CUWHHD_API wp_status wp_unet_destroy(wp_unet* h);

/* ------------------------------------------------------------- batched projection ------- */
/* No reference counterpart: the reference projects one grid per process.  A batch holds `count`
   independent grids of uneven sizes (dims[i] = 2 or 3, extents ext[3*i..3*i+2] (z ignored for 2D),
   uniform spacing dx[i], caller-owned face fractions ax[i], ay[i], az[i] (az may be NULL when all
   grids are 2D)).  Each grid is projected as the reference test does for one grid
   (TestLocalProjection.cpp:666-767): b = -div(a u), a mixed-precision multigrid solve, u <- (u -
   grad p) a, max|div u|, wavelet potential recovery.  wp_batch_run launches the whole batch as ONE
   CUDA graph whose grids are spread over `nstreams` concurrent branches (the graph is captured on the
   first run and again whenever the field pointers change); each grid's solve is a device-side loop
   (a conditional while-node) that stops at params->rel_tol or params->max_cycles on every replay, so
   the step counts follow the input.  wp_batch_plan (optional) runs every grid once eagerly on a
   representative input; its step counts order the grids over the branches, costliest first. */
typedef struct wp_batch wp_batch;
CUWHHD_API wp_status wp_batch_create(wp_batch** h, int count, const int* dims, const int* ext, const double* dx,
                                     const float* const* ax, const float* const* ay, const float* const* az,
                                     const wp_mg_params* params, int nstreams);
/* Synchronous; velocities are read only.  cycles (may be NULL) receives each grid's step count. */
CUWHHD_API wp_status wp_batch_plan(wp_batch* h, const float* const* xv, const float* const* yv, const float* const* zv,
                                   int* cycles, void* stream);
/* Projects every grid in place (xv, yv, zv) and writes the potentials (qx, qy, qz; 2D grids write
   qz only and may pass NULL in zv/qx/qy).  Asynchronous on `stream`. */
CUWHHD_API wp_status wp_batch_run(wp_batch* h, float* const* xv, float* const* yv, float* const* zv, float* const* qx,
                                  float* const* qy, float* const* qz, void* stream);
/* Per grid: max|div u| after projection, the final FP64 relative residual and the V-cycles of the
   last run; any output may be NULL.  Synchronous.  WP_ERR_NOT_CONVERGED when any grid's residual is
   above rel_tol (its loop reached max_cycles or a non-finite residual; all outputs written),
   WP_ERR_DEVICE_WAIT when a bounded device wait gave up. */
CUWHHD_API wp_status wp_batch_results(wp_batch* h, double* max_abs_div, double* rel_residual, int* cycles,
                                      void* stream);
/* How wp_batch_run solves the grids.  WP_BATCH_GRAPH: each grid's solve is its own launches on a
   branch of the graph (a while-node per grid).  WP_BATCH_PERSISTENT: every grid's solve runs in ONE
   persistent kernel inside the graph (one 1024-thread CTA per SM) that takes (grid, level, pass)
   tiles from a device work queue: per grid a program of the phases of one refinement step (first
   sweep from zero, sweeps, residual restriction, the single-CTA coarse cycle, prolongation, the
   sweep that adds to the FP64 iterate, FP64 defect and stopping rule) repeated until the rule stops
   it, the grids advancing independently; the divergence, gradient update, max|div u| and recovery
   of the grids run on the graph's branches before and after it.  Same per-cell arithmetic, same
   results as WP_BATCH_GRAPH (up to the order of the FP64 norm reductions).  tile_cells: cells per
   work-queue tile (0 = 32768).  Needs trilinear V(nu1, nu2) cycles with nu1, nu2 >= 1 from a zero
   start and, per grid, levels whose y extent is a multiple of 4 down to a coarse level of at most
   4096 cells whose pack fits the CTA's shared memory; WP_ERR_UNSUPPORTED otherwise (the mode stays
   as it was).  Every wait of the persistent kernel is bounded (WP_ERR_DEVICE_WAIT from
   wp_batch_results when one gave up). */
#define WP_BATCH_GRAPH 0
#define WP_BATCH_PERSISTENT 1
/* WP_BATCH_AUTO: wp_batch_plan times the persistent solve (its tile tuned when tile_cells is 0) and the
   graph mode's solves on the plan's inputs and runs the faster from then on (the graph mode before a
   plan, and for grids the persistent program does not take). */
#define WP_BATCH_AUTO 2
CUWHHD_API wp_status wp_batch_set_mode(wp_batch* h, int mode, long long tile_cells);
/* The mode the batch runs in (WP_BATCH_GRAPH or WP_BATCH_PERSISTENT; for WP_BATCH_AUTO the plan's
   choice) and the tile (cells per work-queue tile).  With tile_cells 0 in WP_BATCH_PERSISTENT or
   WP_BATCH_AUTO mode the tile is the library's to choose: wp_batch_plan then times the persistent
   solve of the plan's inputs with tiles of 4096, 8192, 16384, 32768 and 65536 cells and keeps the
   fastest.  tuned_ms (may be NULL) receives six timings in ms: those five, then the graph mode's
   solves (WP_BATCH_AUTO only); 0 where not timed. */
CUWHHD_API wp_status wp_batch_get_mode(const wp_batch* h, int* mode, long long* tile_cells, float* tuned_ms);
/* WP_BATCH_PERSISTENT batches: activity counters of the persistent kernel (SM clock cycles summed
   over the CTAs, thread 0 of each), synchronous.  out[0..cap-1] receives the sums since counting was
   last enabled: [0] cycles waiting for a free tile, [1] tiles taken, [2] cycles setting up a tile,
   [3] cycles completing tiles and publishing phases, then for each phase type k = 0..8 (active-cell
   sum, defect, first sweep, sweep, sweep into the FP64 iterate, restriction, prolongation, coarse
   cycle, FP32 copy) [4+2k] its tile cycles and [5+2k] its tiles.  enable 1 clears the sums and counts
   the following runs, 0 stops counting.  WP_ERR_UNSUPPORTED in graph mode. */
#define WP_BATCH_PROFILE_SLOTS 22
CUWHHD_API wp_status wp_batch_profile(wp_batch* h, int enable, double* out, int cap, void* stream);
CUWHHD_API wp_status wp_batch_destroy(wp_batch* h);

#ifdef __cplusplus
}
#endif
#endif
