// wp_gen.cu -- seeded synthetic inputs generated on the device: Gaussian random fields with a
// power-law spectrum as sums of random Fourier modes, and MAC velocity fields u = curl(psi) +
// grad(phi) built from them (the same construction as fields.velocity3d on the host, which uses
// FFT synthesis on the grid instead of a truncated mode sum).  No reference counterpart (the
// reference's generator is uniform noise, TestLocalProjection.cpp:185-221).
//
// A field is f(X) = sum_m A_m cos(2 pi (k_m . X) + phi_m) over integer wave vectors
// 0 < |k_m| <= kmax of one half space, X = (x/nx, y/ny, z/nz) in [0,1)^3; A_m = |k_m|^(slope/2) |g_m|
// with g_m complex Gaussian, scaled so that the field variance sum A_m^2 / 2 equals rms^2.  Modes
// come from a host std::mt19937_64 seeded with `seed`, so a seed gives the same field on any GPU.
#include "wp_common.cuh"

#include <cmath>
#include <random>
#include <vector>

namespace {

struct Mode {
    float kx, ky, kz, ph;  // wave vector and phase in turns
};

std::vector<Mode> make_modes(double slope, double rms, int kmax, std::mt19937_64& rng, std::vector<float>& amp) {
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<Mode> m;
    std::vector<double> a;
    for (int kz = 0; kz <= kmax; ++kz)
        for (int ky = -kmax; ky <= kmax; ++ky)
            for (int kx = -kmax; kx <= kmax; ++kx) {
                if (kz == 0 && (ky < 0 || (ky == 0 && kx <= 0))) continue;  // one of each +-k pair
                const double k2 = (double)kx * kx + (double)ky * ky + (double)kz * kz;
                if (k2 > (double)kmax * kmax) continue;
                const double gr = nd(rng), gi = nd(rng);
                a.push_back(std::pow(k2, slope / 4.0) * std::sqrt(gr * gr + gi * gi));
                m.push_back({(float)kx, (float)ky, (float)kz, (float)(std::atan2(gi, gr) / (2.0 * M_PI))});
            }
    double var = 0.0;
    for (double v : a) var += 0.5 * v * v;
    const double sc = var > 0 ? rms / std::sqrt(var) : 0.0;
    amp.resize(a.size());
    for (size_t i = 0; i < a.size(); ++i) amp[i] = (float)(a[i] * sc);
    return m;
}

// out[(z * ex + x) * ey + y] over an (ex, ey, ez) index box (x, y, z extents), positions
// (x/nx, y/ny, z/nz)
__global__ void __launch_bounds__(256) modes_kernel(float* __restrict__ out, int ex, int ey, int ez, float inx,
                                                    float iny, float inz, const Mode* __restrict__ modes,
                                                    const float* __restrict__ amp, int nm) {
    __shared__ Mode sm[256];
    __shared__ float sa[256];
    const long i = blockIdx.x * 256L + threadIdx.x;
    const long n = (long)ex * ey * ez;
    const int y = (int)(i % ey), x = (int)((i / ey) % ex), z = (int)(i / ((long)ey * ex));
    const float X = x * inx, Y = y * iny, Z = z * inz;
    float acc = 0.f;
    for (int m0 = 0; m0 < nm; m0 += 256) {
        __syncthreads();
        if (m0 + threadIdx.x < nm) {
            sm[threadIdx.x] = modes[m0 + threadIdx.x];
            sa[threadIdx.x] = amp[m0 + threadIdx.x];
        }
        __syncthreads();
        const int cnt = min(256, nm - m0);
        for (int k = 0; k < cnt; ++k) {
            const Mode md = sm[k];
            float t = fmaf(md.kx, X, fmaf(md.ky, Y, fmaf(md.kz, Z, md.ph)));
            t -= floorf(t);
            acc = fmaf(sa[k], __cosf(6.28318530718f * t), acc);
        }
    }
    if (i < n) out[i] = acc;
}

// u = curl(q) + grad(phi) on the MAC faces with zero wall-normal faces (StreamInitial.cpp:87-143
// for the curl of an edge potential).  q arrays: qx (nz+1, nx, ny+1), qy (nz+1, nx+1, ny),
// qz (nz, nx+1, ny+1); phi (nz, nx, ny).
__global__ void __launch_bounds__(256) velocity_kernel(float* __restrict__ xv, float* __restrict__ yv,
                                                       float* __restrict__ zv, const float* __restrict__ qx,
                                                       const float* __restrict__ qy, const float* __restrict__ qz,
                                                       const float* __restrict__ phi, int nx, int ny, int nz) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    const float idx = (float)nx, idy = (float)ny, idz = (float)nz;
    auto QX = [&](int zz, int xx, int yy) { return qx[((long)zz * nx + xx) * (ny + 1) + yy]; };
    auto QY = [&](int zz, int xx, int yy) { return qy[((long)zz * (nx + 1) + xx) * ny + yy]; };
    auto QZ = [&](int zz, int xx, int yy) { return qz[((long)zz * (nx + 1) + xx) * (ny + 1) + yy]; };
    auto PH = [&](int zz, int xx, int yy) { return phi[((long)zz * nx + xx) * ny + yy]; };
    // x faces (z < nz, x <= nx, y < ny)
    if (z < nz && x <= nx && y < ny) {
        float v = 0.f;
        if (x > 0 && x < nx)
            v = (QZ(z, x, y + 1) - QZ(z, x, y)) * idy - (QY(z + 1, x, y) - QY(z, x, y)) * idz +
                (PH(z, x, y) - PH(z, x - 1, y)) * idx;
        xv[((long)z * (nx + 1) + x) * ny + y] = v;
    }
    // y faces (z < nz, x < nx, y <= ny)
    if (z < nz && x < nx && y <= ny) {
        float v = 0.f;
        if (y > 0 && y < ny)
            v = (QX(z + 1, x, y) - QX(z, x, y)) * idz - (QZ(z, x + 1, y) - QZ(z, x, y)) * idx +
                (PH(z, x, y) - PH(z, x, y - 1)) * idy;
        yv[((long)z * nx + x) * (ny + 1) + y] = v;
    }
    // z faces (z <= nz, x < nx, y < ny)
    if (z <= nz && x < nx && y < ny) {
        float v = 0.f;
        if (z > 0 && z < nz)
            v = (QY(z, x + 1, y) - QY(z, x, y)) * idx - (QX(z, x, y + 1) - QX(z, x, y)) * idy +
                (PH(z, x, y) - PH(z - 1, x, y)) * idz;
        zv[((long)z * nx + x) * ny + y] = v;
    }
}

wp_status field_into(float* out, int ex, int ey, int ez, int nx, int ny, int nz, double slope, double rms, int kmax,
                     std::mt19937_64& rng, cudaStream_t s) {
    std::vector<float> amp;
    std::vector<Mode> modes = make_modes(slope, rms, kmax, rng, amp);
    const int nm = (int)modes.size();
    Mode* dm = nullptr;
    float* da = nullptr;
    WP_CUDA_TRY(cudaMallocAsync((void**)&dm, sizeof(Mode) * (nm ? nm : 1), s));
    WP_CUDA_TRY(cudaMallocAsync((void**)&da, sizeof(float) * (nm ? nm : 1), s));
    WP_CUDA_TRY(cudaMemcpyAsync(dm, modes.data(), sizeof(Mode) * nm, cudaMemcpyHostToDevice, s));
    WP_CUDA_TRY(cudaMemcpyAsync(da, amp.data(), sizeof(float) * nm, cudaMemcpyHostToDevice, s));
    const long n = (long)ex * ey * ez;
    WP_KERNEL("random_field", 4.0 * n, s,
              modes_kernel<<<wp_cdiv(n, 256), 256, 0, s>>>(out, ex, ey, ez, 1.f / nx, 1.f / ny, 1.f / nz, dm, da, nm));
    // the host vectors must outlive the copies
    WP_CUDA_TRY(cudaStreamSynchronize(s));
    cudaFreeAsync(dm, s);
    cudaFreeAsync(da, s);
    return WP_OK;
}

}  // namespace

extern "C" CUWHHD_API wp_status wp_random_field3d(float* out, int nx, int ny, int nz, double slope, double rms, int kmax,
                                                  unsigned long long seed, void* stream) {
    if (!out || nx < 1 || ny < 1 || nz < 1 || kmax < 1 || kmax > 32 || !(rms >= 0)) {
        wp_set_error_msg("wp_random_field3d: bad arguments (kmax in [1, 32])");
        return WP_ERR_INVALID_ARG;
    }
    std::mt19937_64 rng(seed);
    return field_into(out, nx, ny, nz, nx, ny, nz, slope, rms, kmax, rng, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_velocity3d(float* xv, float* yv, float* zv, int nx, int ny, int nz,
                                              unsigned long long seed, double psi_slope, double psi_rms,
                                              double phi_slope, double phi_rms, int kmax, void* stream) {
    if (!xv || !yv || !zv || nx < 2 || ny < 2 || nz < 2 || nz >= 65535 || kmax < 1 || kmax > 32) {
        wp_set_error_msg("wp_velocity3d: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nq[3] = {(size_t)(nz + 1) * nx * (ny + 1), (size_t)(nz + 1) * (nx + 1) * ny,
                          (size_t)nz * (nx + 1) * (ny + 1)};
    const size_t np = (size_t)nz * nx * ny;
    float* buf = nullptr;
    WP_CUDA_TRY(cudaMallocAsync((void**)&buf, sizeof(float) * (nq[0] + nq[1] + nq[2] + np), s));
    float* qx = buf;
    float* qy = qx + nq[0];
    float* qz = qy + nq[1];
    float* ph = qz + nq[2];
    std::mt19937_64 rng(seed);
    // (x extent, y extent, z extent) of each staggered array
    wp_status st = field_into(qx, nx, ny + 1, nz + 1, nx, ny, nz, psi_slope, psi_rms, kmax, rng, s);
    if (st == WP_OK) st = field_into(qy, nx + 1, ny, nz + 1, nx, ny, nz, psi_slope, psi_rms, kmax, rng, s);
    if (st == WP_OK) st = field_into(qz, nx + 1, ny + 1, nz, nx, ny, nz, psi_slope, psi_rms, kmax, rng, s);
    if (st == WP_OK) st = field_into(ph, nx, ny, nz, nx, ny, nz, phi_slope, phi_rms, kmax, rng, s);
    if (st == WP_OK) {
        const dim3 g(wp_cdiv(ny + 1, 32), wp_cdiv(nx + 1, 8), nz + 1);
        WP_KERNEL("velocity_assemble", 4.0 * (3.0 * np + nq[0] + nq[1] + nq[2] + np), s,
                  velocity_kernel<<<g, dim3(32, 8), 0, s>>>(xv, yv, zv, qx, qy, qz, ph, nx, ny, nz));
    }
    cudaFreeAsync(buf, s);
    return st;
}
