// wp_dst.cu -- Dirichlet Poisson solve -lap_h p = f by DST-I along x, y and z, in FP64.
//
// Reference behaviour: CuDst3D (cuDst3D.cu:202-341): odd extension into a 2(n+1)-point complex
// FFT per axis (cuFFT), orthonormal scaling sqrt(2/(n+1)), division by the eigenvalues
// sum_i (2 - 2 cos(k_i pi / (n_i + 1))) and the factor dx*dy (cuDstProj_dx, :172-200), then the
// same transforms again (the orthonormal DST-I is its own inverse).
//
// B200 design: no FFT library.  Each axis transform is a dense product with the n x n orthonormal
// DST-I matrix (precomputed once per extent on the host in FP64), applied to a tile of C whole
// lines staged in shared memory (the same tile geometry as the wavelet passes: coalesced along y,
// bank-conflict-free column-parallel inner loop).  For the grid sizes of the coarse and gauge
// solves (n <= a few hundred) the O(n) work per element is cheaper than an FFT's passes.
#include "wp_common.cuh"

#include <cmath>
#include <mutex>
#include <new>
#include <vector>

namespace {

constexpr int NT = 256;

struct Geom {
    long s_in, s_out, pstride;
    int ni;
    int contiguous;
};

template <int C>
__global__ void __launch_bounds__(NT) dst_axis_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                                      const double* __restrict__ M, int N, Geom g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* S = reinterpret_cast<double*>(smem_raw);
    constexpr int CP = C + 1;
    const int tid = threadIdx.x;
    const int i0 = blockIdx.x * C;
    const long obase = (long)blockIdx.y * g.s_out;
    for (int i = tid; i < C * N; i += NT) {
        int col, p;
        if (g.contiguous) { col = i / N; p = i - col * N; }
        else { col = i % C; p = i / C; }
        double v = 0.0;
        if (i0 + col < g.ni) v = src[obase + (long)(i0 + col) * g.s_in + (long)p * g.pstride];
        S[p * CP + col] = v;
    }
    __syncthreads();
    // out[k][col] = sum_j M[k][j] S[j][col]; lanes span columns, warps span k
    constexpr int KPER = NT / C;
    const int col = tid % C, k0 = tid / C;
    for (int k = k0; k < N; k += KPER) {
        double acc = 0.0;
        const double* Mk = M + (long)k * N;
        for (int j = 0; j < N; ++j) acc = fma(__ldg(Mk + j), S[j * CP + col], acc);
        if (i0 + col < g.ni) dst[obase + (long)(i0 + col) * g.s_in + (long)k * g.pstride] = acc;
    }
}

__global__ void __launch_bounds__(256) dst_eig_kernel(double* __restrict__ p, int nx, int ny, int nz, double scale) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (y >= ny || x >= nx) return;
    const double pi = 3.14159265358979323846;
    const double mu = 2.0 - 2.0 * cos((x + 1) * pi / (nx + 1));
    const double nu = 2.0 - 2.0 * cos((y + 1) * pi / (ny + 1));
    const double ku = 2.0 - 2.0 * cos((z + 1) * pi / (nz + 1));
    p[y + (long)x * ny + (long)z * nx * ny] *= scale / (mu + nu + ku);
}

template <int C>
cudaError_t launch_axis(const double* src, double* dst, const double* M, int N, Geom g, int nouter, cudaStream_t s) {
    const size_t smem = (size_t)N * (C + 1) * sizeof(double);
    auto k = dst_axis_kernel<C>;
    cudaError_t e = wp_set_smem(k, smem);
    if (e != cudaSuccess) return e;
    const int tok = wp_prof_start(s);
    k<<<dim3((g.ni + C - 1) / C, nouter), NT, smem, s>>>(src, dst, M, N, g);
    e = cudaGetLastError();
    wp_prof_stop(tok, "dst_axis", 16.0 * N * (double)g.ni * nouter, s);
    return e;
}

cudaError_t apply_axis(const double* src, double* dst, const double* M, int DX, int DY, int DZ, char axis,
                       cudaStream_t s) {
    Geom g;
    int N, nouter;
    if (axis == 'y') { N = DY; g.s_in = DY; g.ni = DX; g.s_out = (long)DX * DY; nouter = DZ; g.pstride = 1; g.contiguous = 1; }
    else if (axis == 'x') { N = DX; g.s_in = 1; g.ni = DY; g.s_out = (long)DX * DY; nouter = DZ; g.pstride = DY; g.contiguous = 0; }
    else { N = DZ; g.s_in = 1; g.ni = DY; g.s_out = DY; nouter = DX; g.pstride = (long)DX * DY; g.contiguous = 0; }
    int C = 32;
    while (C > 4 && (size_t)N * (C + 1) * sizeof(double) > 150 * 1024) C >>= 1;
    if ((size_t)N * (C + 1) * sizeof(double) > 227 * 1024) return cudaErrorInvalidValue;
    switch (C) {
        case 32: return launch_axis<32>(src, dst, M, N, g, nouter, s);
        case 16: return launch_axis<16>(src, dst, M, N, g, nouter, s);
        case 8: return launch_axis<8>(src, dst, M, N, g, nouter, s);
        default: return launch_axis<4>(src, dst, M, N, g, nouter, s);
    }
}

}  // namespace

struct wp_dst3d {
    int n[3];
    double h[3];
    double* M[3];  // orthonormal DST-I matrices per axis
    double* tmp;
};

extern "C" CUWHHD_API wp_status wp_dst3d_create(wp_dst3d** out, int nx, int ny, int nz, double dx, double dy, double dz) {
    if (!out) { wp_set_error_msg("wp_dst3d_create: null handle"); return WP_ERR_INVALID_ARG; }
    *out = nullptr;
    if (nx < 1 || ny < 1 || nz < 1 || nx > 1024 || ny > 1024 || nz > 1024 || nz > 65535 || !(dx > 0) || !(dy > 0) ||
        !(dz > 0)) {
        wp_set_error_msg("wp_dst3d_create: extents must be in [1, 1024] and spacings > 0");
        return WP_ERR_INVALID_ARG;
    }
    wp_dst3d* h = new (std::nothrow) wp_dst3d();
    if (!h) return WP_ERR_INVALID_ARG;
    const int n[3] = {nx, ny, nz};
    const double hs[3] = {dx, dy, dz};
    for (int a = 0; a < 3; ++a) {
        h->n[a] = n[a];
        h->h[a] = hs[a];
        const int m = n[a];
        std::vector<double> M((size_t)m * m);
        const double sc = std::sqrt(2.0 / (m + 1));
        for (int k = 0; k < m; ++k)
            for (int j = 0; j < m; ++j) M[(size_t)k * m + j] = sc * std::sin(M_PI * (double)(j + 1) * (k + 1) / (m + 1));
        cudaError_t e = cudaMalloc((void**)&h->M[a], sizeof(double) * M.size());
        if (e == cudaSuccess) e = cudaMemcpy(h->M[a], M.data(), sizeof(double) * M.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { wp_set_cuda_error(e, "dst3d create", __FILE__, __LINE__); wp_dst3d_destroy(h); return WP_ERR_CUDA; }
    }
    cudaError_t e = cudaMalloc((void**)&h->tmp, sizeof(double) * (size_t)nx * ny * nz);
    if (e != cudaSuccess) { wp_set_cuda_error(e, "dst3d create", __FILE__, __LINE__); wp_dst3d_destroy(h); return WP_ERR_CUDA; }
    *out = h;
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_dst3d_solve(wp_dst3d* h, double* dst, const double* f, void* stream) {
    if (!h || !dst || !f) { wp_set_error_msg("wp_dst3d_solve: null pointer"); return WP_ERR_INVALID_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
    // forward x, y, z; eigen division; inverse z, y, x (ping-pong between dst and tmp)
    cudaError_t e;
    if ((e = apply_axis(f, h->tmp, h->M[0], nx, ny, nz, 'x', s)) != cudaSuccess) goto fail;
    if ((e = apply_axis(h->tmp, dst, h->M[1], nx, ny, nz, 'y', s)) != cudaSuccess) goto fail;
    if ((e = apply_axis(dst, h->tmp, h->M[2], nx, ny, nz, 'z', s)) != cudaSuccess) goto fail;
    {
        const int tok = wp_prof_start(s);
        dst_eig_kernel<<<dim3(wp_cdiv(ny, 32), wp_cdiv(nx, 8), nz), dim3(32, 8), 0, s>>>(h->tmp, nx, ny, nz,
                                                                                       h->h[0] * h->h[1]);
        e = cudaGetLastError();
        wp_prof_stop(tok, "dst_eigen", 16.0 * nx * ny * nz, s);
        if (e != cudaSuccess) goto fail;
    }
    if ((e = apply_axis(h->tmp, dst, h->M[2], nx, ny, nz, 'z', s)) != cudaSuccess) goto fail;
    if ((e = apply_axis(dst, h->tmp, h->M[1], nx, ny, nz, 'y', s)) != cudaSuccess) goto fail;
    if ((e = apply_axis(h->tmp, dst, h->M[0], nx, ny, nz, 'x', s)) != cudaSuccess) goto fail;
    return WP_OK;
fail:
    wp_set_cuda_error(e, "dst3d solve", __FILE__, __LINE__);
    return WP_ERR_CUDA;
}

extern "C" CUWHHD_API wp_status wp_dst3d_destroy(wp_dst3d* h) {
    if (!h) return WP_OK;
    for (int a = 0; a < 3; ++a) if (h->M[a]) cudaFree(h->M[a]);
    if (h->tmp) cudaFree(h->tmp);
    delete h;
    return WP_OK;
}

// ------------------------------------------------------------------ allocation-free variant
// Same transforms as wp_dst3d_solve, with the three DST-I matrices and the ping-pong buffer in a
// file-scope device array instead of handle-owned allocations.  Extents are limited to
// WP_DST_NOALLOC_MAX_EXTENT per axis and WP_DST_NOALLOC_MAX_CELLS cells in total.
namespace {

constexpr int kNoAllocMaxN = WP_DST_NOALLOC_MAX_EXTENT;
constexpr long kNoAllocMaxCells = WP_DST_NOALLOC_MAX_CELLS;
constexpr long kNoAllocWords = 3L * kNoAllocMaxN * kNoAllocMaxN + kNoAllocMaxCells;

// [M_x | M_y | M_z (kNoAllocMaxN^2 doubles each) | tmp (kNoAllocMaxCells doubles)]
static __device__ __align__(256) double g_dst_scratch[kNoAllocWords];

double* g_dst_scratch_ptr[64] = {nullptr};
std::mutex g_dst_scratch_mu;

// M[k][j] = sqrt(2/(m+1)) sin(pi (j+1)(k+1)/(m+1)); the product is reduced modulo 2(m+1) so the
// sinpi argument is exact.
__global__ void dst_matrix_kernel(double* __restrict__ M, int m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m * m) return;
    const int k = i / m, j = i - k * m;
    const long r = ((long)(j + 1) * (k + 1)) % (2L * (m + 1));
    M[i] = sqrt(2.0 / (m + 1)) * sinpi((double)r / (m + 1));
}

// Resolves the scratch address on the current device once (cudaGetSymbolAddress, checked).  The
// address stays valid for the life of the device's primary context: after cudaDeviceReset (or any
// teardown of that context) the cached value is stale, so the entry point is not to be called on
// that device again in the same process.
cudaError_t noalloc_scratch(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_dst_scratch_mu);
    if (!g_dst_scratch_ptr[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, g_dst_scratch);
        if (e != cudaSuccess) return e;
        g_dst_scratch_ptr[dev] = p;
    }
    *out = g_dst_scratch_ptr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" CUWHHD_API wp_status wp_dst3d_solve_noalloc(double* dst, const double* f, int nx, int ny, int nz, double dx,
                                                       double dy, double dz, void* stream) {
    if (!dst || !f) { wp_set_error_msg("wp_dst3d_solve_noalloc: null pointer"); return WP_ERR_INVALID_ARG; }
    if (nx < 1 || ny < 1 || nz < 1 || !(dx > 0) || !(dy > 0) || !(dz > 0)) {
        wp_set_error_msg("wp_dst3d_solve_noalloc: extents must be >= 1 and spacings > 0");
        return WP_ERR_INVALID_ARG;
    }
    if (nx > kNoAllocMaxN || ny > kNoAllocMaxN || nz > kNoAllocMaxN || (long)nx * ny * nz > kNoAllocMaxCells) {
        wp_set_error_msg("wp_dst3d_solve_noalloc: grid exceeds the static scratch (at most 64 per axis and 64^3 "
                         "cells); use wp_dst3d_create/wp_dst3d_solve");
        return WP_ERR_INVALID_ARG;
    }
    double* scratch = nullptr;
    cudaError_t e = noalloc_scratch(&scratch);
    if (e != cudaSuccess) { wp_set_cuda_error(e, "dst3d noalloc scratch address", __FILE__, __LINE__); return WP_ERR_CUDA; }
    cudaStream_t s = (cudaStream_t)stream;
    double* M[3] = {scratch, scratch + (long)kNoAllocMaxN * kNoAllocMaxN, scratch + 2L * kNoAllocMaxN * kNoAllocMaxN};
    double* tmp = scratch + 3L * kNoAllocMaxN * kNoAllocMaxN;
    const int n[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a) {
        const int tok = wp_prof_start(s);
        dst_matrix_kernel<<<wp_cdiv((size_t)n[a] * n[a], 256), 256, 0, s>>>(M[a], n[a]);
        e = cudaGetLastError();
        wp_prof_stop(tok, "dst_matrix", 8.0 * n[a] * n[a], s);
        if (e != cudaSuccess) goto fail;
    }
    if ((e = apply_axis(f, tmp, M[0], nx, ny, nz, 'x', s)) != cudaSuccess) goto fail;
    if ((e = apply_axis(tmp, dst, M[1], nx, ny, nz, 'y', s)) != cudaSuccess) goto fail;
    if ((e = apply_axis(dst, tmp, M[2], nx, ny, nz, 'z', s)) != cudaSuccess) goto fail;
    {
        const int tok = wp_prof_start(s);
        dst_eig_kernel<<<dim3(wp_cdiv(ny, 32), wp_cdiv(nx, 8), nz), dim3(32, 8), 0, s>>>(tmp, nx, ny, nz, dx * dy);
        e = cudaGetLastError();
        wp_prof_stop(tok, "dst_eigen", 16.0 * nx * ny * nz, s);
        if (e != cudaSuccess) goto fail;
    }
    if ((e = apply_axis(tmp, dst, M[2], nx, ny, nz, 'z', s)) != cudaSuccess) goto fail;
    if ((e = apply_axis(dst, tmp, M[1], nx, ny, nz, 'y', s)) != cudaSuccess) goto fail;
    if ((e = apply_axis(tmp, dst, M[0], nx, ny, nz, 'x', s)) != cudaSuccess) goto fail;
    return WP_OK;
fail:
    wp_set_cuda_error(e, "dst3d noalloc solve", __FILE__, __LINE__);
    return WP_ERR_CUDA;
}
