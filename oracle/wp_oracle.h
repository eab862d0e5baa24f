/*
 * wp_oracle.h -- FP64 CPU oracle for the WaveletPotentials projection-and-recovery path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference algorithm used by
 * tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the checker.  The
 * product library (waveletpotentials_b200/csrc) never links or calls it.
 *
 * Array layout follows the reference (Utils.h:46-47, INDEX3D): y is the fastest index,
 * element (x, y, z) of an array with extents (DX, DY, DZ) lives at y + x*DY + z*DX*DY.
 * MAC shapes for an nx*ny*nz grid (TestLocalProjection.cpp:536-542):
 *   xv (nx+1,ny,nz)  yv (nx,ny+1,nz)  zv (nx,ny,nz+1)
 *   qx (nx,ny+1,nz+1) qy (nx+1,ny,nz+1) qz (nx+1,ny+1,nz); 2D qz (nx+1,ny+1).
 */
#ifndef WP_ORACLE_H
#define WP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* wavelet identifiers: same numeric values as the reference enum (WaveletTypes.h:7-27) */
#define OR_CDF3_5 2
#define OR_CDF2_6 5
#define OR_CDF4_4 6
#define OR_CDF4_6 7
#define OR_CDF2_8 10
#define OR_CDF3_7 11
#define OR_CDF2_0 16
#define OR_CDF1_1 17
#define OR_CDF1_7 18

/* one full-depth 1D transform of a line in place (cuWHHDForward.cu:5-105 forward, :349-464 inverse) */
int or_dwt_line(double* line, int n, int levels, int wavelet, char bc, int forward);
/* the same transform applied along one axis of a 3D array (cuWHHDForward.cu:1122-1153) */
int or_dwt_axis(double* a, int DX, int DY, int DZ, int levels, char axis, int wavelet, char bc, int forward);
/* diagonal of the Gram matrix of the synthesis basis, ||B_i||^2 (cuGetInnerProduct.cu:92-126) */
int or_ip_diag(double* out, int dim, int wavelet, char bc);

/* pointwise local projection of velocity coefficients to potential coefficients */
int or_project3d(double* qx, double* qy, double* qz, const double* xv, const double* yv, const double* zv,
                 int nx, int ny, int nz, double dx, double dy, double dz);
int or_project2d(double* qz, const double* xv, const double* yv, int nx, int ny, double dx, double dy);
int or_project2d_nq(double* qz, const double* xv, const double* yv, int nx, int ny, double dx, double dy);
/* the same projection with Dirichlet domain walls (cuProjectLocal_q_3d_nq_ccc) */
int or_project3d_nq(double* qx, double* qy, double* qz, const double* xv, const double* yv, const double* zv,
                    int nx, int ny, int nz, double dx, double dy, double dz);

/* full potential recovery: 9 forward passes, projection, 9 inverse passes (3D, bc 'n' or 'd');
   4 + 1 + 2 (2D) */
int or_recover3d(double* qx, double* qy, double* qz, const double* xv, const double* yv, const double* zv,
                 int nx, int ny, int nz, double dx, double dy, double dz, char bc);
int or_recover2d(double* qz, const double* xv, const double* yv, int nx, int ny, double dx, double dy, char bc);

/* discrete curl of an edge potential onto MAC faces (StreamInitial.cpp:87-175) */
void or_curl3d(double* xv, double* yv, double* zv, const double* qx, const double* qy, const double* qz,
               int nx, int ny, int nz, double dx, double dy, double dz);
void or_curl2d(double* xv, double* yv, const double* qz, int nx, int ny, double dx, double dy);

/* b = -div(a u) on cells (cuConvergence.cu:40-67, :483-500) */
void or_divergence3d(double* b, const double* xv, const double* yv, const double* zv,
                     const double* ax, const double* ay, const double* az, int nx, int ny, int nz,
                     double dx, double dy, double dz);
void or_divergence2d(double* b, const double* xv, const double* yv, const double* ax, const double* ay,
                     int nx, int ny, double dx, double dy);
/* u <- (u - grad p) [* a] with grad p zero on boundary / closed faces (cuGradient.cu:1841-1891) */
void or_grad_subtract3d(double* xv, double* yv, double* zv, const double* p,
                        const double* ax, const double* ay, const double* az, int nx, int ny, int nz,
                        double dx, double dy, double dz, int multiply_frac);
void or_grad_subtract2d(double* xv, double* yv, const double* p, const double* ax, const double* ay,
                        int nx, int ny, double dx, double dy, int multiply_frac);

/* signed distance (positive in fluid) to a union of spheres; face open fractions from it
   (cuSolidLevelSet3D.cu:11-90) */
void or_sdf_spheres3d(double* sdf, int nx, int ny, int nz, double dx, const double* centers, const double* radii,
                      int nspheres);
void or_sdf_boxes3d(double* sdf, int nx, int ny, int nz, double dx, const double* lo, const double* hi, int nboxes);
void or_fractions3d(double* ax, double* ay, double* az, const double* sdf, int nx, int ny, int nz, double dx);
void or_fractions2d(double* ax, double* ay, const double* sdf, int nx, int ny, double dx);

/* fractional multigrid (cuMultigridFrac3D.cu:9-327, cuMultigridFrac2D.cu:28-215), Neumann walls.
   prolong 0: the reference's piecewise-constant prolongation (cuProlongate3D.cu:594-617);
   prolong 1: cell-centred trilinear (bilinear in 2D) prolongation, the convergent variant.
   history (may be NULL) receives ||f - A p|| / ||f|| after each cycle. Returns number of levels. */
int or_mgfrac3d_solve(double* p, const double* p0, const double* f, const double* ax, const double* ay,
                      const double* az, int nx, int ny, int nz, double dx, double dy, double dz,
                      int ncycles, int nu1, int nu2, double omega, int prolong, double* history);
/* face open fractions of an arbitrary level set with 128 x 128 sub-face samples on cut faces
   (CuSolidLevelSet3D::GetFrac(ax, ay, az, ls, dim, dx), cuSolidLevelSet3D.cu:164-372) */
void or_fractions3d_subsampled(double* ax, double* ay, double* az, const double* ls, int nx, int ny, int nz, double dx);
/* eikonal redistancing (CuFastSweeping::Solve, reinit != 0: ReinitLevelSet), in place */
void or_fast_sweep(double* ls, int nx, int ny, int nz, double dx, int iters, int reinit);
/* particles to a level set (CuFastSweeping::ParticlesToLs), xyz: count x 3 positions */
void or_particles_to_ls(double* ls, const double* xyz, int count, int nx, int ny, int nz, double dx, double radius,
                        double max_dis, int iters);
void or_particles_to_ls_narrow(double* ls, const double* xyz, int count, int nx, int ny, int nz, double dx,
                               double radius, int iters);
/* coefficient truncation of a potential, in place (CuWaveletPotentialRecover3D::CutCoefficients,
   cuWaveletPotentialRecover3D.cu:123-239); 1 for a level outside [0, min log2 n] */
int or_cut3d(double* qx, double* qy, double* qz, int nx, int ny, int nz, int level);
/* index-sparse V-cycles (CuMultigridFrac3D::Solve_index, cuMultigridFrac3D.cu:347-420): only cells with
   a face fraction >= 1e-12 are swept, their residuals go to a residual workspace shared by the levels
   (zero at the start) and the restriction reads it for every child; post-smoothing runs nu1 sweeps
   (nu2 unused).  counts (may be NULL) receives the listed cells per level.  Returns the levels. */
int or_mgfrac3d_solve_index(double* p, const double* p0, const double* f, const double* ax, const double* ay,
                            const double* az, int nx, int ny, int nz, double dx, double dy, double dz, int ncycles,
                            int nu1, int nu2, double omega, double* history, long* counts);
int or_mgfrac2d_solve(double* p, const double* p0, const double* f, const double* ax, const double* ay,
                      int nx, int ny, double dx, double dy, int ncycles, int nu1, int nu2, double omega,
                      int prolong, double* history);
/* ||f - A p||_2 / ||f||_2 (cuWeightedJacobi3D.cu:1384-1407); r (may be NULL) receives f - A p */
double or_frac_residual3d(double* r, const double* p, const double* f, const double* ax, const double* ay,
                          const double* az, int nx, int ny, int nz, double dx, double dy, double dz);
double or_frac_residual2d(double* r, const double* p, const double* f, const double* ax, const double* ay,
                          int nx, int ny, double dx, double dy);
/* one weighted-Jacobi sweep (cuWeightedJacobi3D.cu:620-695) */
void or_jacobi3d(double* dst, const double* src, const double* f, const double* ax, const double* ay,
                 const double* az, int nx, int ny, int nz, const double* dxs, const double* dys,
                 const double* dzs, double omega);

/* Dirichlet Poisson solve -lap_h p = f by DST-I in x, y, z (cuDst3D.cu:172-341) */
void or_dst3d_poisson(double* p, const double* f, int nx, int ny, int nz, double dx, double dy, double dz);

/* OpenMP threads of the parallel loops: set (n > 0) / query */
void or_set_threads(int n);
int or_get_threads(void);

#ifdef __cplusplus
}
#endif

#endif
