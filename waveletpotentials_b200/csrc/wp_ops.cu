// wp_ops.cu -- field operators around the solver: divergence, gradient update, max-abs, solid
// level sets and face fractions (3D and 2D).
//
// Reference behaviour: cuGetB_vel_frac_3d(_n) (cuConvergence.cu:40-122; the _n variant computes a
// boundary term it never uses, so both return b = -div(a u)), cuGetB_vel_frac_2d (:483-530),
// cuGradient3D_frac_p_n (cuGradient.cu:1841-1891) followed by CudaMatAdd(-1) / CudaMatMul(a)
// (TestLocalProjection.cpp:672-680), CudaFindMaxValue (cudaMath.cu:1269-1280), cuInitLsSphere /
// cuComputeFrac / cuGetAx,Ay,Az (cuSolidLevelSet3D.cu:11-90).
// All kernels map threadIdx.x to y (the contiguous index) so every access is coalesced.
#include "wp_common.cuh"

#include <algorithm>
#include <map>

#include <cstring>
#include <vector>

namespace {

constexpr float kEps = 1e-12f;

// FRAC = false treats every face as fully open (a = 1): the divergence of an already a-weighted field
template <bool FRAC>
__global__ void __launch_bounds__(256) div3d_kernel(float* __restrict__ b, const float* __restrict__ xv,
                                                    const float* __restrict__ yv, const float* __restrict__ zv,
                                                    const float* __restrict__ ax, const float* __restrict__ ay,
                                                    const float* __restrict__ az, int nx, int ny, int nz, float dxi,
                                                    float dyi, float dzi) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (y >= ny || x >= nx) return;
    const long sxv = (long)(nx + 1) * ny, syv = (long)nx * (ny + 1), szv = (long)nx * ny;
    const long ix = y + (long)x * ny + z * sxv, iy = y + (long)x * (ny + 1) + z * syv, iz = y + (long)x * ny + z * szv;
    float v;
    if (FRAC)
        v = (xv[ix + ny] * ax[ix + ny] - xv[ix] * ax[ix]) * dxi + (yv[iy + 1] * ay[iy + 1] - yv[iy] * ay[iy]) * dyi +
            (zv[iz + szv] * az[iz + szv] - zv[iz] * az[iz]) * dzi;
    else
        v = (xv[ix + ny] - xv[ix]) * dxi + (yv[iy + 1] - yv[iy]) * dyi + (zv[iz + szv] - zv[iz]) * dzi;
    b[iz] = -v;
}

template <bool FRAC>
__global__ void __launch_bounds__(256) div2d_kernel(float* __restrict__ b, const float* __restrict__ xv,
                                                    const float* __restrict__ yv, const float* __restrict__ ax,
                                                    const float* __restrict__ ay, int nx, int ny, float dxi, float dyi) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y;
    if (y >= ny || x >= nx) return;
    const long ix = y + (long)x * ny, iy = y + (long)x * (ny + 1);
    if (FRAC)
        b[ix] = -((xv[ix + ny] * ax[ix + ny] - xv[ix] * ax[ix]) * dxi + (yv[iy + 1] * ay[iy + 1] - yv[iy] * ay[iy]) * dyi);
    else
        b[ix] = -((xv[ix + ny] - xv[ix]) * dxi + (yv[iy + 1] - yv[iy]) * dyi);
}

// u <- (u - grad p) [* a] on all faces; grad p = 0 on wall faces and where a <= eps.  TP = double:
// the pressure is the FP64 iterate and the update is formed in FP64, rounded once when stored.
template <typename TP>
__global__ void __launch_bounds__(256) grad3d_kernel(float* __restrict__ xv, float* __restrict__ yv, float* __restrict__ zv,
                                                     const TP* __restrict__ p, const float* __restrict__ ax,
                                                     const float* __restrict__ ay, const float* __restrict__ az,
                                                     int nx, int ny, int nz, TP gx, TP gy, TP gz, int mul) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    const long sp = (long)nx * ny;
    // x faces: (x in [0,nx], y in [0,ny), z in [0,nz))
    if (y < ny && x <= nx && z < nz) {
        const long i = y + (long)x * ny + (long)z * (nx + 1) * ny;
        const float a = ax[i];
        TP g = 0;
        if (x > 0 && x < nx && a > kEps) {
            const long ip = y + (long)x * ny + z * sp;
            g = (p[ip] - p[ip - ny]) * gx;
        }
        const TP u = (TP)xv[i] - g;
        xv[i] = (float)(mul ? u * (TP)a : u);
    }
    if (y <= ny && x < nx && z < nz) {
        const long i = y + (long)x * (ny + 1) + (long)z * nx * (ny + 1);
        const float a = ay[i];
        TP g = 0;
        if (y > 0 && y < ny && a > kEps) {
            const long ip = y + (long)x * ny + z * sp;
            g = (p[ip] - p[ip - 1]) * gy;
        }
        const TP u = (TP)yv[i] - g;
        yv[i] = (float)(mul ? u * (TP)a : u);
    }
    if (y < ny && x < nx && z <= nz) {
        const long i = y + (long)x * ny + (long)z * sp;
        const float a = az[i];
        TP g = 0;
        if (z > 0 && z < nz && a > kEps) g = (p[i] - p[i - sp]) * gz;
        const TP u = (TP)zv[i] - g;
        zv[i] = (float)(mul ? u * (TP)a : u);
    }
}

__global__ void __launch_bounds__(256) grad2d_kernel(float* __restrict__ xv, float* __restrict__ yv, const float* __restrict__ p,
                                                     const float* __restrict__ ax, const float* __restrict__ ay, int nx,
                                                     int ny, float gx, float gy, int mul) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y;
    if (y < ny && x <= nx) {
        const long i = y + (long)x * ny;
        const float a = ax[i];
        float g = 0.f;
        if (x > 0 && x < nx && a > kEps) g = (p[i] - p[i - ny]) * gx;
        float u = xv[i] - g;
        xv[i] = mul ? u * a : u;
    }
    if (y <= ny && x < nx) {
        const long i = y + (long)x * (ny + 1);
        const float a = ay[i];
        float g = 0.f;
        if (y > 0 && y < ny && a > kEps) {
            const long ip = y + (long)x * ny;
            g = (p[ip] - p[ip - 1]) * gy;
        }
        float u = yv[i] - g;
        yv[i] = mul ? u * a : u;
    }
}

// max |x|: non-negative floats order like their bit patterns
__global__ void __launch_bounds__(256) maxabs_kernel(const float* __restrict__ x, size_t n, unsigned int* out) {
    float m = 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float v = fabsf(x[i]);
        m = (v > m || v != v) ? v : m;  // NaN propagates
    }
    for (int o = 16; o > 0; o >>= 1) {
        float t = __shfl_xor_sync(0xffffffffu, m, o);
        m = (t > m || t != t) ? t : m;
    }
    __shared__ float red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = (red[w] > m || red[w] != red[w]) ? red[w] : m;
        atomicMax(out, __float_as_uint(m));
    }
}

struct Sphere {
    float c[3];
    float r;
};

__global__ void __launch_bounds__(256) sdf_spheres_kernel(float* __restrict__ sdf, int nx, int ny, int nz, float h,
                                                          const Sphere* __restrict__ sp, int count) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (y >= ny || x >= nx) return;
    const float px = (x + 0.5f) * h, py = (y + 0.5f) * h, pz = (z + 0.5f) * h;
    float best = 1e30f;
    for (int s = 0; s < count; ++s) {
        const float dx = px - sp[s].c[0], dy = py - sp[s].c[1], dz = pz - sp[s].c[2];
        best = fminf(best, sqrtf(dx * dx + dy * dy + dz * dz) - sp[s].r);
    }
    sdf[y + (long)x * ny + (long)z * nx * ny] = best;
}

// union with axis-aligned boxes: exact box signed distance, min with the existing level set
struct Box {
    float lo[3], hi[3];
};

__global__ void __launch_bounds__(256) sdf_boxes_kernel(float* __restrict__ sdf, int nx, int ny, int nz, float h,
                                                        const Box* __restrict__ bx, int count) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (y >= ny || x >= nx) return;
    const float p[3] = {(x + 0.5f) * h, (y + 0.5f) * h, (z + 0.5f) * h};
    const long i = y + (long)x * ny + (long)z * nx * ny;
    float best = sdf[i];
    for (int b = 0; b < count; ++b) {
        float out = 0.f, inside = -1e30f;
        for (int c = 0; c < 3; ++c) {
            const float ctr = 0.5f * (bx[b].lo[c] + bx[b].hi[c]), half = 0.5f * (bx[b].hi[c] - bx[b].lo[c]);
            const float q = fabsf(p[c] - ctr) - half;
            if (q > 0.f) out += q * q;
            inside = fmaxf(inside, q);
        }
        best = fminf(best, sqrtf(out) + fminf(inside, 0.f));
    }
    sdf[i] = best;
}

__global__ void __launch_bounds__(256) sdf_circles_kernel(float* __restrict__ sdf, int nx, int ny, float h,
                                                          const Sphere* __restrict__ sp, int count) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y;
    if (y >= ny || x >= nx) return;
    const float px = (x + 0.5f) * h, py = (y + 0.5f) * h;
    float best = 1e30f;
    for (int s = 0; s < count; ++s) {
        const float dx = px - sp[s].c[0], dy = py - sp[s].c[1];
        best = fminf(best, sqrtf(dx * dx + dy * dy) - sp[s].r);
    }
    sdf[y + (long)x * ny] = best;
}

__device__ __forceinline__ float frac_from_ls(float h, float l, float r) {
    const float dif = r - l;
    const float d = sqrtf(fmaxf(h * h - dif * dif, 1e-14f));
    return 1.f - fminf(fmaxf((1.f - (r + l) / d) * 0.5f, 0.f), 1.f);
}

__global__ void __launch_bounds__(256) frac3d_kernel(float* __restrict__ ax, float* __restrict__ ay, float* __restrict__ az,
                                                     const float* __restrict__ ls, int nx, int ny, int nz, float h) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    const long s = (long)nx * ny;
    if (y < ny && x <= nx && z < nz) {
        const int xl = max(x - 1, 0), xr = min(x, nx - 1);
        ax[y + (long)x * ny + (long)z * (nx + 1) * ny] = frac_from_ls(h, ls[y + (long)xl * ny + z * s], ls[y + (long)xr * ny + z * s]);
    }
    if (y <= ny && x < nx && z < nz) {
        const int yl = max(y - 1, 0), yr = min(y, ny - 1);
        ay[y + (long)x * (ny + 1) + (long)z * nx * (ny + 1)] = frac_from_ls(h, ls[yl + (long)x * ny + z * s], ls[yr + (long)x * ny + z * s]);
    }
    if (y < ny && x < nx && z <= nz) {
        const int zl = max(z - 1, 0), zr = min(z, nz - 1);
        az[y + (long)x * ny + (long)z * s] = frac_from_ls(h, ls[y + (long)x * ny + zl * s], ls[y + (long)x * ny + zr * s]);
    }
}

__global__ void __launch_bounds__(256) frac2d_kernel(float* __restrict__ ax, float* __restrict__ ay,
                                                     const float* __restrict__ ls, int nx, int ny, float h) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y;
    if (y < ny && x <= nx) {
        const int xl = max(x - 1, 0), xr = min(x, nx - 1);
        ax[y + (long)x * ny] = frac_from_ls(h, ls[y + (long)xl * ny], ls[y + (long)xr * ny]);
    }
    if (y <= ny && x < nx) {
        const int yl = max(y - 1, 0), yr = min(y, ny - 1);
        ay[y + (long)x * (ny + 1)] = frac_from_ls(h, ls[yl + (long)x * ny], ls[yr + (long)x * ny]);
    }
}

}  // namespace

extern "C" CUWHHD_API wp_status wp_divergence_frac3d(float* b, const float* xv, const float* yv, const float* zv,
                                                     const float* ax, const float* ay, const float* az, int nx, int ny,
                                                     int nz, double dx, double dy, double dz, void* stream) {
    const bool frac = ax || ay || az;
    if (!b || !xv || !yv || !zv || (frac && (!ax || !ay || !az)) || nx <= 0 || ny <= 0 || nz <= 0 || nz > 65535) {
        wp_set_error_msg("wp_divergence_frac3d: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    dim3 grid(wp_cdiv(ny, 32), wp_cdiv(nx, 8), nz);
    const float dxi = (float)(1.0 / dx), dyi = (float)(1.0 / dy), dzi = (float)(1.0 / dz);
    cudaStream_t s = (cudaStream_t)stream;
    const double faces = (double)(nx + 1) * ny * nz * 3, cells = (double)nx * ny * nz;
    if (frac)
        WP_KERNEL("divergence", 4.0 * (2 * faces + cells), s,
                  div3d_kernel<true><<<grid, dim3(32, 8), 0, s>>>(b, xv, yv, zv, ax, ay, az, nx, ny, nz, dxi, dyi, dzi));
    else
        WP_KERNEL("divergence", 4.0 * (faces + cells), s,
                  div3d_kernel<false><<<grid, dim3(32, 8), 0, s>>>(b, xv, yv, zv, ax, ay, az, nx, ny, nz, dxi, dyi, dzi));
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_divergence_frac2d(float* b, const float* xv, const float* yv, const float* ax,
                                                     const float* ay, int nx, int ny, double dx, double dy, void* stream) {
    const bool frac = ax || ay;
    if (!b || !xv || !yv || (frac && (!ax || !ay)) || nx <= 0 || ny <= 0) {
        wp_set_error_msg("wp_divergence_frac2d: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    dim3 grid(wp_cdiv(ny, 32), wp_cdiv(nx, 8));
    cudaStream_t s = (cudaStream_t)stream;
    const float dxi = (float)(1.0 / dx), dyi = (float)(1.0 / dy);
    const double faces = 2.0 * (nx + 1) * ny, cells = (double)nx * ny;
    if (frac)
        WP_KERNEL("divergence2d", 4.0 * (2 * faces + cells), s,
                  div2d_kernel<true><<<grid, dim3(32, 8), 0, s>>>(b, xv, yv, ax, ay, nx, ny, dxi, dyi));
    else
        WP_KERNEL("divergence2d", 4.0 * (faces + cells), s,
                  div2d_kernel<false><<<grid, dim3(32, 8), 0, s>>>(b, xv, yv, ax, ay, nx, ny, dxi, dyi));
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_grad_subtract_frac3d(float* xv, float* yv, float* zv, const float* p, const float* ax,
                                                        const float* ay, const float* az, int nx, int ny, int nz,
                                                        double dx, double dy, double dz, int multiply_frac, void* stream) {
    if (!xv || !yv || !zv || !p || !ax || !ay || !az || nx <= 0 || ny <= 0 || nz <= 0 || nz >= 65535) {
        wp_set_error_msg("wp_grad_subtract_frac3d: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    dim3 grid(wp_cdiv(ny + 1, 32), wp_cdiv(nx + 1, 8), nz + 1);
    // (p_r - p_l) / (dx_l + dx_r) * 2 with uniform spacing (cuGradient.cu:1862)
    cudaStream_t s = (cudaStream_t)stream;
    const double faces = (double)(nx + 1) * ny * nz * 3, cells = (double)nx * ny * nz;
    WP_KERNEL("grad_subtract", 4.0 * (3 * faces + cells), s,
              grad3d_kernel<float><<<grid, dim3(32, 8), 0, s>>>(xv, yv, zv, p, ax, ay, az, nx, ny, nz,
                                                                (float)(2.0 / (dx + dx)), (float)(2.0 / (dy + dy)),
                                                                (float)(2.0 / (dz + dz)), multiply_frac));
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_grad_subtract_frac3d_p64(float* xv, float* yv, float* zv, const double* p,
                                                            const float* ax, const float* ay, const float* az, int nx,
                                                            int ny, int nz, double dx, double dy, double dz,
                                                            int multiply_frac, void* stream) {
    if (!xv || !yv || !zv || !p || !ax || !ay || !az || nx <= 0 || ny <= 0 || nz <= 0 || nz >= 65535) {
        wp_set_error_msg("wp_grad_subtract_frac3d_p64: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    dim3 grid(wp_cdiv(ny + 1, 32), wp_cdiv(nx + 1, 8), nz + 1);
    cudaStream_t s = (cudaStream_t)stream;
    const double faces = (double)(nx + 1) * ny * nz * 3, cells = (double)nx * ny * nz;
    WP_KERNEL("grad_subtract", 4.0 * 3 * faces + 8.0 * cells, s,
              grad3d_kernel<double><<<grid, dim3(32, 8), 0, s>>>(xv, yv, zv, p, ax, ay, az, nx, ny, nz, 2.0 / (dx + dx),
                                                                 2.0 / (dy + dy), 2.0 / (dz + dz), multiply_frac));
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_grad_subtract_frac2d(float* xv, float* yv, const float* p, const float* ax, const float* ay,
                                                        int nx, int ny, double dx, double dy, int multiply_frac, void* stream) {
    if (!xv || !yv || !p || !ax || !ay || nx <= 0 || ny <= 0) { wp_set_error_msg("wp_grad_subtract_frac2d: bad arguments"); return WP_ERR_INVALID_ARG; }
    dim3 grid(wp_cdiv(ny + 1, 32), wp_cdiv(nx + 1, 8));
    cudaStream_t s = (cudaStream_t)stream;
    WP_KERNEL("grad_subtract2d", 4.0 * (6.0 * (nx + 1) * ny + (double)nx * ny), s,
              grad2d_kernel<<<grid, dim3(32, 8), 0, s>>>(xv, yv, p, ax, ay, nx, ny, (float)(2.0 / (dx + dx)),
                                                         (float)(2.0 / (dy + dy)), multiply_frac));
    return WP_OK;
}

wp_status wp_max_abs_device(const float* x, size_t n, unsigned int* d_out, cudaStream_t s) {
    WP_CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(unsigned int), s));
    if (n == 0) return WP_OK;
    unsigned blocks = wp_cdiv(n, 256);
    const unsigned cap = (unsigned)wp_sm_count() * 8;
    if (blocks > cap) blocks = cap;
    WP_KERNEL("max_abs", 4.0 * n, s, maxabs_kernel<<<blocks, 256, 0, s>>>(x, n, d_out));
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_max_abs(const float* x, size_t n, double* out, void* stream) {
    if ((!x && n) || !out) { wp_set_error_msg("wp_max_abs: null pointer"); return WP_ERR_INVALID_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    // one device word per (host thread, device), allocated on first use: no allocation per call
    thread_local std::map<int, unsigned int*> slots;
    int dev = 0;
    WP_CUDA_TRY(cudaGetDevice(&dev));
    unsigned int*& d = slots[dev];
    if (!d) WP_CUDA_TRY(cudaMalloc((void**)&d, sizeof(unsigned int)));
    wp_status st = wp_max_abs_device(x, n, d, s);
    unsigned int bits = 0;
    if (st == WP_OK) {
        const cudaError_t e = wp_read_small(&bits, d, sizeof(bits), s);
        if (e != cudaSuccess) { wp_set_cuda_error(e, "wp_max_abs", __FILE__, __LINE__); st = WP_ERR_CUDA; }
    }
    float f;
    memcpy(&f, &bits, sizeof(f));
    *out = (double)f;
    return st;
}

extern "C" CUWHHD_API wp_status wp_sdf_spheres3d(float* sdf, int nx, int ny, int nz, double dx, const double* centers,
                                                 const double* radii, int count, void* stream) {
    if (!sdf || nx <= 0 || ny <= 0 || nz <= 0 || count < 0 || (count > 0 && (!centers || !radii)) || count > 4096) {
        wp_set_error_msg("wp_sdf_spheres3d: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<Sphere> hs(count > 0 ? count : 1);
    for (int i = 0; i < count; ++i) {
        hs[i].c[0] = (float)centers[3 * i];
        hs[i].c[1] = (float)centers[3 * i + 1];
        hs[i].c[2] = (float)centers[3 * i + 2];
        hs[i].r = (float)radii[i];
    }
    Sphere* d = nullptr;
    WP_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(Sphere) * hs.size(), s));
    WP_CUDA_TRY(cudaMemcpyAsync(d, hs.data(), sizeof(Sphere) * hs.size(), cudaMemcpyHostToDevice, s));
    dim3 grid(wp_cdiv(ny, 32), wp_cdiv(nx, 8), nz);
    const int tok = wp_prof_start(s);
    sdf_spheres_kernel<<<grid, dim3(32, 8), 0, s>>>(sdf, nx, ny, nz, (float)dx, d, count);
    cudaError_t e = cudaGetLastError();
    wp_prof_stop(tok, "sdf_spheres", 4.0 * nx * ny * nz, s);
    // the host staging vector must outlive the async copy
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaFreeAsync(d, s);
    if (e != cudaSuccess || e2 != cudaSuccess) { wp_set_cuda_error(e != cudaSuccess ? e : e2, "sdf", __FILE__, __LINE__); return WP_ERR_CUDA; }
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_fractions3d(float* ax, float* ay, float* az, const float* sdf, int nx, int ny, int nz,
                                               double dx, void* stream) {
    if (!ax || !ay || !az || !sdf || nx <= 0 || ny <= 0 || nz <= 0 || nz >= 65535) { wp_set_error_msg("wp_fractions3d: bad arguments"); return WP_ERR_INVALID_ARG; }
    dim3 grid(wp_cdiv(ny + 1, 32), wp_cdiv(nx + 1, 8), nz + 1);
    cudaStream_t s = (cudaStream_t)stream;
    WP_KERNEL("fractions", 4.0 * (4.0 * nx * ny * nz), s,
              frac3d_kernel<<<grid, dim3(32, 8), 0, s>>>(ax, ay, az, sdf, nx, ny, nz, (float)dx));
    return WP_OK;
}

// ------------------------------------------------ subsampled face fractions of a level set
// CuSolidLevelSet3D::GetFrac(ax, ay, az, ls, dim, dx) (cuSolidLevelSet3D.cu:356-372) with the kernels
// cuGetAx/Ay/Az_divide (:164-316): the level set interpolated quadratically at the face centre
// (InterpolateQuadratic3D, Interpolation.cuh:119-156) decides open (> dx), closed (<= -dx) or cut;
// a cut face is the share of 128 x 128 sub-face samples where the trilinear interpolant
// (InterpolateLinear3D with cuGetIxFx's clamping, Interpolation.cuh:16-29, 80-117) is positive.
// FP64 arithmetic in the reference's term order (its default build); the level set is FP32.
// Work split: one thread per face classifies and lists the cut faces; one warp per listed face
// counts its samples (16 rounds of 32 lanes x 32 samples with ballots).
namespace {
constexpr double kClampL = (double)1e-10f;  // CLAMP_L of the double build (Interpolation.cuh:9)

__device__ __forceinline__ double ls_at(const float* __restrict__ ls, int x, int y, int z, int nx, int ny) {
    return (double)ls[y + (long)x * ny + (long)z * nx * ny];
}

__device__ double ls_quadratic(const float* __restrict__ ls, double x, double y, double z, int nx, int ny, int nz) {
    const int ix = (int)floor(x - 0.5), iy = (int)floor(y - 0.5), iz = (int)floor(z - 0.5);
    const double fx = x - ix, fy = y - iy, fz = z - iz;
    auto p2 = [](double v) { return v * v; };
    const double wx[3] = {0.5 * p2(1.5 - fx), 0.75 - p2(fx - 1.0), 0.5 * p2(fx - 0.5)};
    const double wy[3] = {0.5 * p2(1.5 - fy), 0.75 - p2(fy - 1.0), 0.5 * p2(fy - 0.5)};
    const double wz[3] = {0.5 * p2(1.5 - fz), 0.75 - p2(fz - 1.0), 0.5 * p2(fz - 0.5)};
    double r = 0.0;
    for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                const int xx = min(max(ix + j, 0), nx - 1), yy = min(max(iy + i, 0), ny - 1);
                const int zz = min(max(iz + k, 0), nz - 1);
                r += wx[j] * wy[i] * wz[k] * ls_at(ls, xx, yy, zz, nx, ny);
            }
    return r;
}

__device__ __forceinline__ void clamp_index(int& i, double& f, double x, int n) {
    x = fmax(kClampL, x);
    i = (int)x;
    if (i >= n - 1) {
        i = n - 2;
        f = 1.0;  // 1.f - CLAMP_L evaluates in float to 1
    } else {
        f = x - i;
    }
}

__device__ double ls_linear(const float* __restrict__ ls, double x, double y, double z, int nx, int ny, int nz) {
    int ix, iy, iz;
    double fx, fy, fz;
    clamp_index(ix, fx, x, nx);
    clamp_index(iy, fy, y, ny);
    clamp_index(iz, fz, z, nz);
    const double wx0 = 1 - fx, wy0 = 1 - fy, wz0 = 1 - fz;
    double r = ls_at(ls, ix, iy, iz, nx, ny) * wx0 * wy0 * wz0;
    r += ls_at(ls, ix, iy + 1, iz, nx, ny) * wx0 * fy * wz0;
    r += ls_at(ls, ix + 1, iy, iz, nx, ny) * fx * wy0 * wz0;
    r += ls_at(ls, ix + 1, iy + 1, iz, nx, ny) * fx * fy * wz0;
    r += ls_at(ls, ix, iy, iz + 1, nx, ny) * wx0 * wy0 * fz;
    r += ls_at(ls, ix, iy + 1, iz + 1, nx, ny) * wx0 * fy * fz;
    r += ls_at(ls, ix + 1, iy, iz + 1, nx, ny) * fx * wy0 * fz;
    r += ls_at(ls, ix + 1, iy + 1, iz + 1, nx, ny) * fx * fy * fz;
    return r;
}

// face (axis a, index i of that axis' face array) -> its integer coordinates
__device__ __forceinline__ void face_coords(int a, long i, int nx, int ny, int& x, int& y, int& z) {
    const int ex = nx + (a == 0), ey = ny + (a == 1);
    y = (int)(i % ey);
    const long xz = i / ey;
    x = (int)(xz % ex);
    z = (int)(xz / ex);
}

__global__ void frac_classify_kernel(float* __restrict__ ax, float* __restrict__ ay, float* __restrict__ az,
                                     const float* __restrict__ ls, int nx, int ny, int nz, double dx,
                                     unsigned* __restrict__ work, unsigned* __restrict__ nwork) {
    const long n0 = (long)(nx + 1) * ny * nz, n1 = (long)nx * (ny + 1) * nz, n2 = (long)nx * ny * (nz + 1);
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n0 + n1 + n2; t += (long)gridDim.x * blockDim.x) {
        const int a = t < n0 ? 0 : (t < n0 + n1 ? 1 : 2);
        const long i = t - (a == 0 ? 0 : (a == 1 ? n0 : n0 + n1));
        int x, y, z;
        face_coords(a, i, nx, ny, x, y, z);
        const double inv = 1.0 / dx;
        const double px = (a == 0 ? (double)x : x + 0.5) * dx, py = (a == 1 ? (double)y : y + 0.5) * dx;
        const double pz = (a == 2 ? (double)z : z + 0.5) * dx;
        const double v = ls_quadratic(ls, px * inv - 0.5, py * inv - 0.5, pz * inv - 0.5, nx, ny, nz);
        float* out = a == 0 ? ax : (a == 1 ? ay : az);
        if (v > dx) {
            out[i] = 1.f;
        } else if (v > -dx) {
            out[i] = 0.f;
            work[atomicAdd(nwork, 1u)] = ((unsigned)a << 30) | (unsigned)i;
        } else {
            out[i] = 0.f;
        }
    }
}

__global__ void __launch_bounds__(256) frac_subsample_kernel(float* __restrict__ ax, float* __restrict__ ay,
                                                             float* __restrict__ az, const float* __restrict__ ls,
                                                             int nx, int ny, int nz, double dx,
                                                             const unsigned* __restrict__ work,
                                                             const unsigned* __restrict__ nwork) {
    const int lane = threadIdx.x & 31;
    const unsigned total = *nwork;
    const unsigned warps = gridDim.x * (blockDim.x >> 5);
    const double inv = 1.0 / dx, dsub = dx / 128, half = 0.5 * dsub;
    for (unsigned w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < total; w += warps) {
        const unsigned code = work[w];
        const int a = (int)(code >> 30);
        const long i = code & 0x3fffffffu;
        int x, y, z;
        face_coords(a, i, nx, ny, x, y, z);
        // the two in-face axes: u is the reference's inner loop, w its outer loop
        const double fixed = (a == 0 ? x : (a == 1 ? y : z)) * dx;
        const double ub = (a == 0 ? y : x) * dx + half;  // ax: i over y, k over z; ay: j over x, k over z;
        const double wb = (a == 2 ? y : z) * dx + half;  // az: i over y (inner), j over x (outer)
        int count = 0;
        for (int s0 = 0; s0 < 128 * 128; s0 += 32) {
            const int s = s0 + lane;
            const int outer = s >> 7, inner = s & 127;
            double px, py, pz;
            if (a == 0) {
                px = fixed; py = ub + inner * dsub; pz = wb + outer * dsub;
            } else if (a == 1) {
                px = ub + inner * dsub; py = fixed; pz = wb + outer * dsub;
            } else {
                px = ub + outer * dsub; py = wb + inner * dsub; pz = fixed;
            }
            const double v = ls_linear(ls, px * inv - 0.5, py * inv - 0.5, pz * inv - 0.5, nx, ny, nz);
            count += __popc(__ballot_sync(0xffffffffu, v > 0.0));
        }
        if (lane == 0) {
            float* out = a == 0 ? ax : (a == 1 ? ay : az);
            const double r = count * (1.0 / 16384.0);
            out[i] = (float)fmin(fmax(r, 0.0), 1.0);
        }
    }
}
}  // namespace

extern "C" CUWHHD_API wp_status wp_fractions3d_subsampled(float* ax, float* ay, float* az, const float* ls, int nx,
                                                          int ny, int nz, double dx, void* stream) {
    if (!ax || !ay || !az || !ls || nx < 2 || ny < 2 || nz < 2 || !(dx > 0) ||
        (double)(nx + 1) * (ny + 1) * (nz + 1) >= (double)(1u << 30)) {
        wp_set_error_msg("wp_fractions3d_subsampled: bad arguments (extents >= 2, fewer than 2^30 faces per axis, dx > 0)");
        return WP_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const long faces = (long)(nx + 1) * ny * nz + (long)nx * (ny + 1) * nz + (long)nx * ny * (nz + 1);
    unsigned* buf = nullptr;
    WP_CUDA_TRY(cudaMallocAsync((void**)&buf, sizeof(unsigned) * (faces + 1), s));
    cudaError_t e = cudaMemsetAsync(buf, 0, sizeof(unsigned), s);
    if (e == cudaSuccess) {
        const int tok = wp_prof_start(s);
        const unsigned g = (unsigned)std::min<long>(wp_cdiv(faces, 256), (long)wp_sm_count() * 16);
        frac_classify_kernel<<<g, 256, 0, s>>>(ax, ay, az, ls, nx, ny, nz, dx, buf + 1, buf);
        e = cudaGetLastError();
        wp_prof_stop(tok, "frac_classify", 4.0 * faces + 27.0 * 4.0 * faces, s);
    }
    if (e == cudaSuccess) {
        const int tok = wp_prof_start(s);
        frac_subsample_kernel<<<wp_sm_count() * 8, 256, 0, s>>>(ax, ay, az, ls, nx, ny, nz, dx, buf + 1, buf);
        e = cudaGetLastError();
        wp_prof_stop(tok, "frac_subsample", 0.0, s);
    }
    cudaFreeAsync(buf, s);
    if (e != cudaSuccess) { wp_set_cuda_error(e, "subsampled fractions", __FILE__, __LINE__); return WP_ERR_CUDA; }
    return WP_OK;
}

// ------------------------------------------------------------ fast sweeping (eikonal)
// CuFastSweeping::Solve / ReinitLevelSet (cuFastSweeping.cu:215-257, 383-396): a cell whose value
// is above -1e-12 takes the upwind (Godunov) solution of |grad d| = 1 from the smaller neighbour of
// each axis (solve_eikonal_nomin, :98-140; a missing neighbour counts 1e8); cells at or below
// -1e-12 stay fixed and act as the sources.  The reference updates the array in place from
// concurrently running threads, so its iterates depend on scheduling; here each iteration reads
// the previous iterate and writes the other buffer (deterministic, one cell of propagation per
// iteration), which reaches the same fixed point.
namespace {
__device__ double eikonal_upwind(double mx, double my, double mz, double h) {
    double m[3] = {mx, my, mz};
    for (int i = 1; i < 3; ++i)
        for (int j = 0; j < 3 - i; ++j)
            if (m[j] > m[j + 1]) { const double t = m[j]; m[j] = m[j + 1]; m[j + 1] = t; }
    const double d2 = h * h;
    double r = m[0] + h;
    if (r > m[1]) {
        const double s = sqrt(-m[0] * m[0] + 2 * m[0] * m[1] - m[1] * m[1] + d2 + d2);
        r = (m[1] * d2 + m[0] * d2 + h * h * s) / (d2 + d2);
        if (r > m[2]) {
            const double a = sqrt(-m[0] * m[0] * d2 - m[0] * m[0] * d2 + 2 * m[0] * m[1] * d2 - m[1] * m[1] * d2 -
                                  m[1] * m[1] * d2 + 2 * m[0] * m[2] * d2 - m[2] * m[2] * d2 - m[2] * m[2] * d2 +
                                  2 * m[1] * m[2] * d2 + d2 * d2 + d2 * d2 + d2 * d2);
            r = (m[2] * d2 * d2 + m[1] * d2 * d2 + m[0] * d2 * d2 + h * h * h * a) / (d2 * d2 + d2 * d2 + d2 * d2);
        }
    }
    return r;
}

__global__ void fsweep_kernel(float* __restrict__ out, const float* __restrict__ in, int nx, int ny, int nz,
                              double h) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (y >= ny || x >= nx) return;
    const long sl = (long)nx * ny, i = y + (long)x * ny + z * sl;
    const double c = in[i];
    if (!(c > -1e-12)) { out[i] = (float)c; return; }
    const double big = 1e8;
    const double l = x > 0 ? in[i - ny] : big, r = x < nx - 1 ? in[i + ny] : big;
    const double u = y < ny - 1 ? in[i + 1] : big, d = y > 0 ? in[i - 1] : big;
    const double f = z > 0 ? in[i - sl] : big, b = z < nz - 1 ? in[i + sl] : big;
    out[i] = (float)eikonal_upwind(fmin(l, r), fmin(u, d), fmin(f, b), h);
}

__global__ void negate_kernel(float* __restrict__ v, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[i] = -v[i];
}

wp_status fsweep_iters(float* ls, float* tmp, int nx, int ny, int nz, double h, int iters, cudaStream_t s) {
    const dim3 g(wp_cdiv(ny, 32), wp_cdiv(nx, 8), nz);
    const double bytes = 8.0 * nx * ny * nz;
    float* a = ls;
    float* b = tmp;
    for (int k = 0; k < iters; ++k) {
        WP_KERNEL("fast_sweep", bytes, s, fsweep_kernel<<<g, dim3(32, 8), 0, s>>>(b, a, nx, ny, nz, h));
        std::swap(a, b);
    }
    if (a != ls) WP_CUDA_TRY(cudaMemcpyAsync(ls, a, sizeof(float) * (size_t)nx * ny * nz, cudaMemcpyDeviceToDevice, s));
    return WP_OK;
}

wp_status fsweep_entry(float* ls, int nx, int ny, int nz, double dx, int iters, bool reinit, cudaStream_t s) {
    if (!ls || nx < 1 || ny < 1 || nz < 1 || nz > 65535 || !(dx > 0) || iters < 0) {
        wp_set_error_msg("wp_fast_sweep: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    const long n = (long)nx * ny * nz;
    float* tmp = nullptr;
    WP_CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * n, s));
    const unsigned gn = (unsigned)std::min<long>(wp_cdiv(n, 256), (long)wp_sm_count() * 16);
    wp_status st = WP_OK;
    auto neg = [&]() -> wp_status {
        WP_KERNEL("negate", 8.0 * n, s, negate_kernel<<<gn, 256, 0, s>>>(ls, n));
        return WP_OK;
    };
    if (reinit) {
        if ((st = neg()) == WP_OK && (st = fsweep_iters(ls, tmp, nx, ny, nz, dx, iters, s)) == WP_OK &&
            (st = neg()) == WP_OK)
            st = fsweep_iters(ls, tmp, nx, ny, nz, dx, iters, s);
    } else {
        st = fsweep_iters(ls, tmp, nx, ny, nz, dx, iters, s);
    }
    cudaFreeAsync(tmp, s);
    return st;
}
}  // namespace

// CuFastSweeping::ParticlesToLs (cuFastSweeping.cu:259-349): every cell starts at dx; each particle
// lowers the 8 cells around it to (distance to the particle) - radius (a float minimum, order
// independent); then the sign is flipped outside / the inside set to max_dis, swept, flipped back
// and swept again, and the result negated.  Cells the reference would index outside the grid (a
// particle within half a cell of a wall) are skipped here.
namespace {
__device__ __forceinline__ void atomic_min_float(float* a, float v) {
    if (v >= 0.f) atomicMin(reinterpret_cast<int*>(a), __float_as_int(v));
    else atomicMax(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
}

__global__ void particles_rough_kernel(float* __restrict__ ls, const float* __restrict__ xyz, int count, int nx,
                                       int ny, int nz, double dx, double radius) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    const double inv = 1.0 / dx;
    const double x = xyz[3 * p] * inv - 0.5, y = xyz[3 * p + 1] * inv - 0.5, z = xyz[3 * p + 2] * inv - 0.5;
    const int ix = (int)floor(x), iy = (int)floor(y), iz = (int)floor(z);
    const double fx = x - ix, fy = y - iy, fz = z - iz;
    const double wx[2] = {fx * fx, (1.0 - fx) * (1.0 - fx)}, wy[2] = {fy * fy, (1.0 - fy) * (1.0 - fy)};
    const double wz[2] = {fz * fz, (1.0 - fz) * (1.0 - fz)};
    for (int k = 0; k < 2; ++k)
        for (int j = 0; j < 2; ++j)
            for (int i = 0; i < 2; ++i) {
                const int cx = ix + j, cy = iy + i, cz = iz + k;
                if (cx < 0 || cx >= nx || cy < 0 || cy >= ny || cz < 0 || cz >= nz) continue;
                const double d = sqrt(wx[j] + wy[i] + wz[k]) * dx - radius;
                atomic_min_float(ls + cy + (long)cx * ny + (long)cz * nx * ny, (float)d);
            }
}

__global__ void fill_kernel(float* __restrict__ v, long n, float val) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[i] = val;
}

// cuInvLevelSet (cuFastSweeping.cu:302-317): outside (> 0) negated, the rest set to max_dis
__global__ void inv_ls_kernel(float* __restrict__ v, long n, float max_dis) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        v[i] = v[i] > 0.f ? -v[i] : max_dis;
}
}  // namespace

extern "C" CUWHHD_API wp_status wp_particles_to_ls(float* ls, const float* xyz, int count, int nx, int ny, int nz,
                                                   double dx, double radius, double max_dis, int n_iters,
                                                   void* stream) {
    if (!ls || (count > 0 && !xyz) || count < 0 || nx < 1 || ny < 1 || nz < 1 || nz > 65535 || !(dx > 0) ||
        n_iters < 0) {
        wp_set_error_msg("wp_particles_to_ls: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const long n = (long)nx * ny * nz;
    const unsigned gn = (unsigned)std::min<long>(wp_cdiv(n, 256), (long)wp_sm_count() * 16);
    WP_KERNEL("fill", 4.0 * n, s, fill_kernel<<<gn, 256, 0, s>>>(ls, n, (float)dx));
    if (count > 0)
        WP_KERNEL("particles_rough", 12.0 * count, s,
                  particles_rough_kernel<<<(unsigned)wp_cdiv(count, 256), 256, 0, s>>>(ls, xyz, count, nx, ny, nz, dx,
                                                                                     radius));
    float* tmp = nullptr;
    WP_CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * n, s));
    wp_status st = WP_OK;
    // every launch reports through a lambda, so a failed one still reaches the scratch release below
    auto inv = [&]() -> wp_status {
        WP_KERNEL("inv_ls", 8.0 * n, s, inv_ls_kernel<<<gn, 256, 0, s>>>(ls, n, (float)max_dis));
        return WP_OK;
    };
    auto negate = [&]() -> wp_status {
        WP_KERNEL("negate", 8.0 * n, s, negate_kernel<<<gn, 256, 0, s>>>(ls, n));
        return WP_OK;
    };
    if ((st = inv()) == WP_OK && (st = fsweep_iters(ls, tmp, nx, ny, nz, dx, n_iters, s)) == WP_OK &&
        (st = inv()) == WP_OK && (st = fsweep_iters(ls, tmp, nx, ny, nz, dx, n_iters, s)) == WP_OK)
        st = negate();
    cudaFreeAsync(tmp, s);
    return st;
}

// CuFastSweeping::ParticlesToLsNarrow (cuFastSweeping.cu:352-385): the caller's ls is the start (no
// fill); the particles lower it, then n_iters sweeps, negation (cuInvLevelSet_nb), n_iters sweeps, and
// no final negation; max_dis is accepted and unused, as in the reference.
extern "C" CUWHHD_API wp_status wp_particles_to_ls_narrow(float* ls, const float* xyz, int count, int nx, int ny,
                                                          int nz, double dx, double radius, double max_dis,
                                                          int n_iters, void* stream) {
    (void)max_dis;
    if (!ls || (count > 0 && !xyz) || count < 0 || nx < 1 || ny < 1 || nz < 1 || nz > 65535 || !(dx > 0) ||
        n_iters < 0) {
        wp_set_error_msg("wp_particles_to_ls_narrow: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const long n = (long)nx * ny * nz;
    const unsigned gn = (unsigned)std::min<long>(wp_cdiv(n, 256), (long)wp_sm_count() * 16);
    if (count > 0)
        WP_KERNEL("particles_rough", 12.0 * count, s,
                  particles_rough_kernel<<<(unsigned)wp_cdiv(count, 256), 256, 0, s>>>(ls, xyz, count, nx, ny, nz, dx,
                                                                                     radius));
    float* tmp = nullptr;
    WP_CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * n, s));
    wp_status st = WP_OK;
    auto negate = [&]() -> wp_status {
        WP_KERNEL("negate", 8.0 * n, s, negate_kernel<<<gn, 256, 0, s>>>(ls, n));
        return WP_OK;
    };
    if ((st = fsweep_iters(ls, tmp, nx, ny, nz, dx, n_iters, s)) == WP_OK && (st = negate()) == WP_OK)
        st = fsweep_iters(ls, tmp, nx, ny, nz, dx, n_iters, s);
    cudaFreeAsync(tmp, s);
    return st;
}

extern "C" CUWHHD_API wp_status wp_fast_sweep_solve(float* ls, int nx, int ny, int nz, double dx, int n_iters,
                                                    void* stream) {
    return fsweep_entry(ls, nx, ny, nz, dx, n_iters, false, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_fast_sweep_reinit(float* ls, int nx, int ny, int nz, double dx, int n_iters,
                                                     void* stream) {
    return fsweep_entry(ls, nx, ny, nz, dx, n_iters, true, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_sdf_boxes3d(float* sdf, int nx, int ny, int nz, double dx, const double* lo,
                                               const double* hi, int count, void* stream) {
    if (!sdf || nx <= 0 || ny <= 0 || nz <= 0 || nz > 65535 || count < 0 || count > 4096 ||
        (count > 0 && (!lo || !hi))) {
        wp_set_error_msg("wp_sdf_boxes3d: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    if (count == 0) return WP_OK;
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<Box> hb(count);
    for (int i = 0; i < count; ++i)
        for (int c = 0; c < 3; ++c) { hb[i].lo[c] = (float)lo[3 * i + c]; hb[i].hi[c] = (float)hi[3 * i + c]; }
    Box* d = nullptr;
    WP_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(Box) * count, s));
    WP_CUDA_TRY(cudaMemcpyAsync(d, hb.data(), sizeof(Box) * count, cudaMemcpyHostToDevice, s));
    const int tok = wp_prof_start(s);
    sdf_boxes_kernel<<<dim3(wp_cdiv(ny, 32), wp_cdiv(nx, 8), nz), dim3(32, 8), 0, s>>>(sdf, nx, ny, nz, (float)dx, d, count);
    cudaError_t e = cudaGetLastError();
    wp_prof_stop(tok, "sdf_boxes", 8.0 * nx * ny * nz, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaFreeAsync(d, s);
    if (e != cudaSuccess || e2 != cudaSuccess) { wp_set_cuda_error(e != cudaSuccess ? e : e2, "sdf boxes", __FILE__, __LINE__); return WP_ERR_CUDA; }
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_sdf_circles2d(float* sdf, int nx, int ny, double dx, const double* centers,
                                                 const double* radii, int count, void* stream) {
    if (!sdf || nx <= 0 || ny <= 0 || count < 0 || count > 4096 || (count > 0 && (!centers || !radii))) {
        wp_set_error_msg("wp_sdf_circles2d: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<Sphere> hs(count > 0 ? count : 1);
    for (int i = 0; i < count; ++i) {
        hs[i].c[0] = (float)centers[2 * i];
        hs[i].c[1] = (float)centers[2 * i + 1];
        hs[i].c[2] = 0.f;
        hs[i].r = (float)radii[i];
    }
    Sphere* d = nullptr;
    WP_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(Sphere) * hs.size(), s));
    WP_CUDA_TRY(cudaMemcpyAsync(d, hs.data(), sizeof(Sphere) * hs.size(), cudaMemcpyHostToDevice, s));
    const int tok = wp_prof_start(s);
    sdf_circles_kernel<<<dim3(wp_cdiv(ny, 32), wp_cdiv(nx, 8)), dim3(32, 8), 0, s>>>(sdf, nx, ny, (float)dx, d, count);
    cudaError_t e = cudaGetLastError();
    wp_prof_stop(tok, "sdf_circles", 4.0 * nx * ny, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaFreeAsync(d, s);
    if (e != cudaSuccess || e2 != cudaSuccess) { wp_set_cuda_error(e != cudaSuccess ? e : e2, "sdf circles", __FILE__, __LINE__); return WP_ERR_CUDA; }
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_fractions2d(float* ax, float* ay, const float* sdf, int nx, int ny, double dx,
                                               void* stream) {
    if (!ax || !ay || !sdf || nx <= 0 || ny <= 0) { wp_set_error_msg("wp_fractions2d: bad arguments"); return WP_ERR_INVALID_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    WP_KERNEL("fractions2d", 4.0 * 3.0 * nx * ny, s,
              frac2d_kernel<<<dim3(wp_cdiv(ny + 1, 32), wp_cdiv(nx + 1, 8)), dim3(32, 8), 0, s>>>(ax, ay, sdf, nx, ny,
                                                                                               (float)dx));
    return WP_OK;
}
