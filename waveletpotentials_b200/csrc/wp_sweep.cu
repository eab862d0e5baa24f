// wp_sweep.cu -- vector-potential recovery by sweeping and a DST-I gauge projection: the
// reference's comparison baseline for the wavelet recovery (CuParallelSweep3D, cuParallelSweep3D.cu).
//
// Solve (bc 'n', cuParallelSweep3D.cu:939-966): qz = 0; qx and qy start from 0 on the z = 0 plane and
// integrate yv (+dz) and xv (-dz) along z (SweepingQx / SweepingQy, :28-66); the top plane is then
// made tangential-free: qp = the x-integral of qx's top plane (cuSweepingQ_x, :9-26), the top planes
// of qx and qy are cleared and qz's top plane gets -qp / dz (CudaMatAdd, cudaMath.cu:110-118).
// Solve with bc 'd' (SetQxQyBoundary, :925-937): qx's z = 0 plane is 0, qy's is the x-integral of
// zv's bottom face (SweepingQy_x, :68-85); the same z integrals; no top-plane step.
// Project (bc 'n' -> ProjectZero, :1043-1081): b = -div q on the (n-1)^3 interior nodes
// (cuGetB_q_zero_3d, cuConvergence.cu:126-159), the DST-I Poisson solve, and q -= grad phi with
// phi = 0 on the boundary nodes (cuGradientMinus3D_zero_Q, cuGradient.cu:2353-2405, with its spacing
// for the three wall edges).  Project with bc 'd' (ProjectD, :1084-1098) is not built: the reference's
// run of it at 16^3 raised an illegal address.  2D Solve (SweepingQz_x_0, :106-124): qz =
// -x-integral of yv; with bc 'd' (SweepingQz_y then SweepingQz_x, :87-143) the x = 0 column is first
// the y-integral of xv's x = 0 column.
//
// B200 design: the z integrals are column scans, HBM bound (one read of u, one write of q).  A CTA
// takes 32 consecutive y columns (128-byte rows) and splits z into 8 chunks over its 8 warps: chunk
// sums, a prefix over the chunks in shared memory, then each chunk rewritten with its running sum
// (the second read of u hits L2).  The x integral of the top plane is one warp per y row (chunk sums
// and a shuffle scan).  The divergence and the gradient are pointwise; the Poisson solve is the
// library's FP64 DST (wp_dst3d).
#include "wp_common.cuh"

#include <new>

namespace {

constexpr int kChunks = 8;

// out[col + z so] for z = 1 .. nzin: out[col] (plane 0, kept) + s * sum of in[col + z' si], z' < z.
// so = si = ncx ncy (0: that default) scans upward; negative strides scan downward from the base plane.
__global__ void __launch_bounds__(256) sweep_scan_kernel(float* __restrict__ out, const float* __restrict__ in,
                                                         int ncx, int ncy, int nzin, float s, long so = 0,
                                                         long si = 0) {
    __shared__ float part[kChunks][32];
    const int c = threadIdx.x, k = threadIdx.y;
    const int y = blockIdx.x * 32 + c, x = blockIdx.y;
    const bool ok = y < ncy && x < ncx;
    if (so == 0) so = (long)ncx * ncy;
    if (si == 0) si = (long)ncx * ncy;
    const long col = y + (long)x * ncy;
    const int cz = (nzin + kChunks - 1) / kChunks;
    const int z0 = min(k * cz, nzin), z1 = min(z0 + cz, nzin);
    float loc = 0.f;
    if (ok)
        for (int z = z0; z < z1; ++z) loc += in[col + z * si] * s;
    part[k][c] = loc;
    __syncthreads();
    if (ok) {
        float run = out[col];
        for (int j = 0; j < k; ++j) run += part[j][c];
        for (int z = z0; z < z1; ++z) {
            run += in[col + z * si] * s;
            out[col + (z + 1) * so] = run;
        }
    }
}

// bc 'n' top plane: one warp per y row of qx's plane z = nz: qp[x] = dx * sum_{x' < x} qx_top[x'],
// qz[plane nz - 1][x] += qp[x] * mdz (mdz = -1 / dz), x = 0 .. nx
__global__ void sweep_top_kernel(const float* __restrict__ qx, float* __restrict__ qz, int nx, int ny, int nz,
                                 float dx, float mdz) {
    const int row = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    const int ny1 = ny + 1;
    if (row >= ny1) return;
    const float* src = qx + (long)nz * nx * ny1 + row;
    float* dst = qz + (long)(nz - 1) * (nx + 1) * ny1 + row;
    const int per = (nx + 31) / 32;
    const int x0 = min(lane * per, nx), x1 = min(x0 + per, nx);
    float loc = 0.f;
    for (int x = x0; x < x1; ++x) loc += src[(long)x * ny1] * dx;
    float incl = loc;
    for (int o = 1; o < 32; o <<= 1) {
        const float t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    float run = incl - loc;
    for (int x = x0; x < x1; ++x) {
        dst[(long)x * ny1] += run * mdz;
        run += src[(long)x * ny1] * dx;
    }
    if (x0 < x1 && x1 == nx) dst[(long)nx * ny1] += run * mdz;
}

// b = -div q on the interior nodes (x, y, z) = (j + 1, i + 1, k + 1), FP32 as cuGetB_q_zero_3d
__global__ void __launch_bounds__(256) sweep_div_kernel(double* __restrict__ b, const float* __restrict__ qx,
                                                        const float* __restrict__ qy, const float* __restrict__ qz,
                                                        int nx, int ny, int nz, float dxi, float dyi, float dzi) {
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
    const int px = nx - 1, py = ny - 1;
    if (i >= py || j >= px) return;
    const long sqx = (long)nx * (ny + 1), sqy = (long)(nx + 1) * ny, sqz = (long)(nx + 1) * (ny + 1);
    const long qxl = (i + 1) + (long)j * (ny + 1) + (long)(k + 1) * sqx, qxr = qxl + (ny + 1);
    const long qyb = i + (long)(j + 1) * ny + (long)(k + 1) * sqy, qyt = qyb + 1;
    const long qzf = (i + 1) + (long)(j + 1) * (ny + 1) + (long)k * sqz, qzb = qzf + sqz;
    const float v = -((qx[qxr] - qx[qxl]) * dxi + (qy[qyt] - qy[qyb]) * dyi + (qz[qzb] - qz[qzf]) * dzi);
    b[i + (long)j * py + (long)k * px * py] = (double)v;
}

// q -= grad phi, phi = 0 outside the interior nodes; per node the three edges towards +x, +y, +z and,
// on the first interior plane of each axis, the wall edge (cuGradientMinus3D_zero_Q's arithmetic)
__global__ void __launch_bounds__(256) sweep_grad_kernel(float* __restrict__ qx, float* __restrict__ qy,
                                                         float* __restrict__ qz, const double* __restrict__ phi, int nx,
                                                         int ny, int nz, float dxi, float dyi, float dzi) {
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
    const int px = nx - 1, py = ny - 1, pz = nz - 1;
    if (i >= py || j >= px) return;
    const long sp = (long)px * py;
    const long idx = i + (long)j * py + (long)k * sp;
    const int qxy = ny + 1, qyy = ny, qzy = ny + 1;
    const long sqx = (long)qxy * nx, sqy = (long)qyy * (nx + 1), sqz = (long)qzy * (nx + 1);
    const long iqx = (i + 1) + (long)(j + 1) * qxy + (long)(k + 1) * sqx;
    const long iqy = (i + 1) + (long)(j + 1) * qyy + (long)(k + 1) * sqy;
    const long iqz = (i + 1) + (long)(j + 1) * qzy + (long)(k + 1) * sqz;
    const float p = (float)phi[idx];
    const float pdx = p * dxi, pdy = p * dyi, pdz = p * dzi;
    if (i == 0) qy[iqy - 1] -= pdx;
    if (j == 0) qx[iqx - qxy] -= pdy;
    if (k == 0) qz[iqz - sqz] -= pdz;
    float gy = -pdy, gx = -pdx, gz = -pdz;
    if (i < py - 1) gy += (float)phi[idx + 1] * dyi;
    if (j < px - 1) gx += (float)phi[idx + py] * dxi;
    if (k < pz - 1) gz += (float)phi[idx + sp] * dzi;
    qy[iqy] -= gy;
    qx[iqx] -= gx;
    qz[iqz] -= gz;
}

}  // namespace

struct wp_sweep3d {
    int n[3];
    double h[3];
    char bc;
    wp_dst3d* dst;
    double* phi;  // (n - 1)^3 interior nodes
};

extern "C" CUWHHD_API wp_status wp_sweep3d_create(wp_sweep3d** out, int nx, int ny, int nz, double dx, double dy,
                                                  double dz, char bc) {
    if (!out) { wp_set_error_msg("wp_sweep3d_create: null handle"); return WP_ERR_INVALID_ARG; }
    *out = nullptr;
    if (bc != 'n' && bc != 'd') { wp_set_error_msg("wp_sweep3d_create: bc must be 'n' or 'd'"); return WP_ERR_UNSUPPORTED; }
    if (nx < 2 || ny < 2 || nz < 2 || !(dx > 0) || !(dy > 0) || !(dz > 0)) {
        wp_set_error_msg("wp_sweep3d_create: extents must be >= 2 and spacings > 0");
        return WP_ERR_INVALID_ARG;
    }
    wp_sweep3d* h = new (std::nothrow) wp_sweep3d();
    if (!h) return WP_ERR_INVALID_ARG;
    h->n[0] = nx; h->n[1] = ny; h->n[2] = nz;
    h->h[0] = dx; h->h[1] = dy; h->h[2] = dz;
    h->bc = bc;
    // the DST-I gauge projection is the bc 'n' Project's (ProjectZero); bc 'd' handles only solve
    wp_status st = bc == 'n' ? wp_dst3d_create(&h->dst, nx - 1, ny - 1, nz - 1, dx, dy, dz) : WP_OK;
    if (st == WP_OK && bc == 'n') {
        const cudaError_t e = cudaMalloc((void**)&h->phi, sizeof(double) * (size_t)(nx - 1) * (ny - 1) * (nz - 1));
        if (e != cudaSuccess) { wp_set_cuda_error(e, "sweep3d create", __FILE__, __LINE__); st = WP_ERR_CUDA; }
    }
    if (st != WP_OK) { wp_sweep3d_destroy(h); return st; }
    *out = h;
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_sweep3d_solve(wp_sweep3d* h, float* qx, float* qy, float* qz, const float* xv,
                                                 const float* yv, const float* zv, void* stream) {
    if (!h || !qx || !qy || !qz || !xv || !yv || (h->bc == 'd' && !zv)) {
        wp_set_error_msg("wp_sweep3d_solve: null pointer");
        return WP_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
    const long sqx = (long)nx * (ny + 1), sqy = (long)(nx + 1) * ny, nqz = (long)(nx + 1) * (ny + 1) * nz;
    WP_CUDA_TRY(cudaMemsetAsync(qz, 0, sizeof(float) * nqz, s));
    WP_CUDA_TRY(cudaMemsetAsync(qx, 0, sizeof(float) * sqx, s));
    WP_CUDA_TRY(cudaMemsetAsync(qy, 0, sizeof(float) * sqy, s));
    if (h->bc == 'd') {
        // qy's z = 0 plane ((nx+1) rows of ny): row 0 stays 0, row x = x-integral of zv's bottom face
        WP_KERNEL("sweep_x", 8.0 * nx * ny, s,
                  sweep_scan_kernel<<<dim3(wp_cdiv(ny, 32), 1), dim3(32, kChunks), 0, s>>>(qy, zv, 1, ny, nx,
                                                                                         (float)h->h[0]));
    }
    const float dz = (float)h->h[2];
    WP_KERNEL("sweep_z", 8.0 * sqx * nz, s,
              sweep_scan_kernel<<<dim3(wp_cdiv(ny + 1, 32), nx), dim3(32, kChunks), 0, s>>>(qx, yv, nx, ny + 1, nz, dz));
    WP_KERNEL("sweep_z", 8.0 * sqy * nz, s,
              sweep_scan_kernel<<<dim3(wp_cdiv(ny, 32), nx + 1), dim3(32, kChunks), 0, s>>>(qy, xv, nx + 1, ny, nz,
                                                                                          -dz));
    if (h->bc == 'd') return WP_OK;
    // bc 'n': qp from qx's top plane into qz's top plane, then the top planes of qx and qy cleared
    WP_KERNEL("sweep_top", 12.0 * (nx + 1) * (ny + 1), s,
              sweep_top_kernel<<<wp_cdiv((long)(ny + 1) * 32, 256), 256, 0, s>>>(qx, qz, nx, ny, nz, (float)h->h[0],
                                                                               -1.f / dz));
    WP_CUDA_TRY(cudaMemsetAsync(qx + sqx * nz, 0, sizeof(float) * sqx, s));
    WP_CUDA_TRY(cudaMemsetAsync(qy + sqy * nz, 0, sizeof(float) * sqy, s));
    return WP_OK;
}

// CuParallelSweep3D::SolveFromMid (cuParallelSweep3D.cu:967-984): the integrals of Solve run both ways
// from the plane mid_z (and, for qy's plane there, from the row mid_x); mid_y is unused, as in the
// reference.  Any bc.
extern "C" CUWHHD_API wp_status wp_sweep3d_solve_from_mid(wp_sweep3d* h, float* qx, float* qy, float* qz,
                                                          const float* xv, const float* yv, const float* zv, int mid_x,
                                                          int mid_y, int mid_z, void* stream) {
    (void)mid_y;
    if (!h || !qx || !qy || !qz || !xv || !yv || !zv) {
        wp_set_error_msg("wp_sweep3d_solve_from_mid: null pointer");
        return WP_ERR_INVALID_ARG;
    }
    const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
    if (mid_x < 0 || mid_x > nx || mid_z < 0 || mid_z > nz) {
        wp_set_error_msg("wp_sweep3d_solve_from_mid: mid_x must lie in [0, nx] and mid_z in [0, nz]");
        return WP_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const long sqx = (long)nx * (ny + 1), sqy = (long)(nx + 1) * ny, szv = (long)nx * ny;
    const float dx = (float)h->h[0], dz = (float)h->h[2];
    WP_CUDA_TRY(cudaMemsetAsync(qz, 0, sizeof(float) * (size_t)(nx + 1) * (ny + 1) * nz, s));
    WP_CUDA_TRY(cudaMemsetAsync(qx + mid_z * sqx, 0, sizeof(float) * sqx, s));
    // qy's plane mid_z: rows x of ny, from row mid_x = 0 both ways along x with zv's plane mid_z
    float* qp = qy + mid_z * sqy;
    const float* zp = zv + mid_z * szv;
    WP_CUDA_TRY(cudaMemsetAsync(qp + (long)mid_x * ny, 0, sizeof(float) * ny, s));
    const dim3 gy(wp_cdiv(ny, 32), 1), blk(32, kChunks);
    if (mid_x < nx)
        WP_KERNEL("sweep_x", 8.0 * (nx - mid_x) * ny, s,
                  sweep_scan_kernel<<<gy, blk, 0, s>>>(qp + (long)mid_x * ny, zp + (long)mid_x * ny, 1, ny, nx - mid_x,
                                                       dx, ny, ny));
    if (mid_x > 0)
        WP_KERNEL("sweep_x", 8.0 * mid_x * ny, s,
                  sweep_scan_kernel<<<gy, blk, 0, s>>>(qp + (long)mid_x * ny, zp + (long)(mid_x - 1) * ny, 1, ny, mid_x,
                                                       -dx, -ny, -ny));
    // z both ways from plane mid_z: qx with +yv dz, qy with -xv dz (signs flip downward)
    if (mid_z < nz) {
        WP_KERNEL("sweep_z", 8.0 * sqx * (nz - mid_z), s,
                  sweep_scan_kernel<<<dim3(wp_cdiv(ny + 1, 32), nx), blk, 0, s>>>(qx + mid_z * sqx, yv + mid_z * sqx, nx,
                                                                                 ny + 1, nz - mid_z, dz));
        WP_KERNEL("sweep_z", 8.0 * sqy * (nz - mid_z), s,
                  sweep_scan_kernel<<<dim3(wp_cdiv(ny, 32), nx + 1), blk, 0, s>>>(qy + mid_z * sqy, xv + mid_z * sqy,
                                                                                 nx + 1, ny, nz - mid_z, -dz));
    }
    if (mid_z > 0) {
        WP_KERNEL("sweep_z", 8.0 * sqx * mid_z, s,
                  sweep_scan_kernel<<<dim3(wp_cdiv(ny + 1, 32), nx), blk, 0, s>>>(qx + mid_z * sqx,
                                                                                 yv + (mid_z - 1) * sqx, nx, ny + 1,
                                                                                 mid_z, -dz, -sqx, -sqx));
        WP_KERNEL("sweep_z", 8.0 * sqy * mid_z, s,
                  sweep_scan_kernel<<<dim3(wp_cdiv(ny, 32), nx + 1), blk, 0, s>>>(qy + mid_z * sqy,
                                                                                 xv + (mid_z - 1) * sqy, nx + 1, ny,
                                                                                 mid_z, dz, -sqy, -sqy));
    }
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_sweep3d_project(wp_sweep3d* h, float* qx, float* qy, float* qz, void* stream) {
    if (!h || !qx || !qy || !qz) { wp_set_error_msg("wp_sweep3d_project: null pointer"); return WP_ERR_INVALID_ARG; }
    if (h->bc != 'n') {
        wp_set_error_msg("wp_sweep3d_project: bc 'd' (the reference's ProjectD) is not built");
        return WP_ERR_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
    const float dxi = (float)(1.0 / h->h[0]), dyi = (float)(1.0 / h->h[1]), dzi = (float)(1.0 / h->h[2]);
    const dim3 g(wp_cdiv(ny - 1, 32), wp_cdiv(nx - 1, 8), nz - 1);
    const double nodes = (double)(nx - 1) * (ny - 1) * (nz - 1);
    WP_KERNEL("sweep_div", nodes * (24.0 + 8.0), s,
              sweep_div_kernel<<<g, dim3(32, 8), 0, s>>>(h->phi, qx, qy, qz, nx, ny, nz, dxi, dyi, dzi));
    wp_status st = wp_dst3d_solve(h->dst, h->phi, h->phi, stream);
    if (st != WP_OK) return st;
    WP_KERNEL("sweep_grad", nodes * (8.0 + 24.0), s,
              sweep_grad_kernel<<<g, dim3(32, 8), 0, s>>>(qx, qy, qz, h->phi, nx, ny, nz, dxi, dyi, dzi));
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_sweep3d_destroy(wp_sweep3d* h) {
    if (!h) return WP_OK;
    if (h->dst) wp_dst3d_destroy(h->dst);
    if (h->phi) cudaFree(h->phi);
    delete h;
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_sweep2d_solve(float* qz, const float* xv, const float* yv, int nx, int ny, double dx,
                                                 double dy, char bc, void* stream) {
    if (!qz || !yv || nx < 1 || ny < 1 || !(dx > 0) || (bc == 'd' && (!xv || !(dy > 0)))) {
        wp_set_error_msg("wp_sweep2d_solve: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    if (bc != 'n' && bc != 'd') { wp_set_error_msg("wp_sweep2d_solve: bc must be 'n' or 'd'"); return WP_ERR_UNSUPPORTED; }
    cudaStream_t s = (cudaStream_t)stream;
    // qz (nx+1) x (ny+1): x is the outer index, so the x integral is a scan over "planes" of ny+1 rows
    WP_CUDA_TRY(cudaMemsetAsync(qz, 0, sizeof(float) * (ny + 1), s));
    if (bc == 'd') {
        // the x = 0 column: qz(0, y) = qz(0, y - 1) + xv(0, y - 1) dy from qz(0, 0) = 0 (a scan over ny
        // "planes" of one entry)
        WP_KERNEL("sweep_y2d", 8.0 * ny, s,
                  sweep_scan_kernel<<<dim3(1, 1), dim3(32, kChunks), 0, s>>>(qz, xv, 1, 1, ny, (float)dy));
    }
    WP_KERNEL("sweep_x2d", 8.0 * (double)nx * (ny + 1), s,
              sweep_scan_kernel<<<dim3(wp_cdiv(ny + 1, 32), 1), dim3(32, kChunks), 0, s>>>(qz, yv, 1, ny + 1, nx,
                                                                                         -(float)dx));
    return WP_OK;
}
