// wp_recover.cu -- local divergence-free projection in wavelet space and the potential-recovery
// pipelines (3D and 2D).
//
// Reference behaviour:
//   3D projection cuProjectLocal_q_3d_dq_ccc (cuDivLocalProject3D.cu:4013-4246), launched by
//   CuDivLocalProject3D::ProjectLocal_q_ccc (:5273-5308); the wall bc 'n' makes the div-wavelet
//   bc 'd' so this is the kernel on the configured path.  Coefficient index (x,y,z) in [0,n)^3
//   reads xv(x+1,y,z), yv(x,y+1,z), zv(x,y,z+1), writes qx(x,y+1,z+1), qy(x+1,y,z+1), qz(x+1,y+1,z):
//   interior q = (s x v)/|s|^2 with s_i = 4/(dx_i (2^j_i + 1e-12)), j_i = L_i - bitlen(i) + 1;
//   faces (one index 0): a one-component ratio weighted by the inner-product tables
//   (ip_proj = ||B||^2 of CDF3.7 'n' on n points, ip_base = ||B||^2 of CDF4.6 'd' on n+1 points);
//   edges and corner: 0.  Every other q entry is 0.
//   2D projection cuProjectLocal_q_single (cuDivLocalProject.cu:765-1045): both of its passes
//   evaluate the same pointwise ratio (the neighbour terms it computes are unused), so
//   qz(i+1,j+1) = P(i,j) for i,j >= 1 and qz = 0 on the rows/columns 0 and 1.
//   Pipelines CuWaveletPotentialRecover3D::Solve (cuWaveletPotentialRecover3D.cu:16-61) and
//   CuWaveletPotentialRecover2D::Solve (cuWaveletPotentialRecover2D.cu:16-36).
#include "wp_common.cuh"

#include <algorithm>

#include <cmath>
#include <cstdlib>
#include <new>
#include <vector>

wp_status wp_ip_diag_device(double* d_out, int dim, int wavelet, char bc, cudaStream_t s);
wp_status wp_ip_gram01_device(double* d_out, int dim, int wavelet, char bc, cudaStream_t s);

namespace {

constexpr float kEps = 1e-12f;

// per-axis table of length n: [scale s_i | ip_proj[i] | ip_base[i+1]]
struct AxisTab {
    const float* s;
    const float* ip0;
    const float* ip1;
};

// project3d_kernel's per-coefficient body: coefficient (x, y, z) with its velocity coefficients
// already loaded
__device__ __forceinline__ void project3d_cell(float* __restrict__ qx, float* __restrict__ qy, float* __restrict__ qz,
                                               int nx, int ny, int x, int y, int z, float xin, float yin, float zin,
                                               const AxisTab& tx, const AxisTab& ty, const AxisTab& tz) {
    const long sqx = (long)nx * (ny + 1), sqy = (long)(nx + 1) * ny, sqz = (long)(nx + 1) * (ny + 1);
    const float sx = tx.s[x], sy = ty.s[y], sz = tz.s[z];
    float oX = 0.f, oY = 0.f, oZ = 0.f;
    if (x > 0 && y > 0 && z > 0) {
        const float inv = 1.f / (sy * sy + sx * sx + sz * sz);
        oZ = (sy * xin - sx * yin) * inv;
        oX = (sz * yin - sy * zin) * inv;
        oY = (sx * zin - sz * xin) * inv;
    } else {
        const float ip0x = tx.ip0[x], ip1x = tx.ip1[x], ip0y = ty.ip0[y], ip1y = ty.ip1[y];
        const float ip0z = tz.ip0[z], ip1z = tz.ip1[z];
        if (x == 0 && y > 0 && z > 0) {
            const float szByBz = sz * ip0x * ip1y * ip0z, syByBz = sy * ip0x * ip0y * ip1z;
            oX = (yin * szByBz - zin * syByBz) / (sy * syByBz + sz * szByBz + kEps);
        } else if (y == 0 && x > 0 && z > 0) {
            const float sxBxBz = sx * ip0x * ip0y * ip1z, szBxBz = sz * ip1x * ip0y * ip0z;
            oY = (zin * sxBxBz - xin * szBxBz) / (sx * sxBxBz + sz * szBxBz + kEps);
        } else if (z == 0 && x > 0 && y > 0) {
            const float syBxBy = sy * ip1x * ip0y * ip0z, sxBxBy = sx * ip0x * ip1y * ip0z;
            oZ = (xin * syBxBy - yin * sxBxBy) / (sx * sxBxBy + sy * syBxBy + kEps);
        }
    }
    qx[(y + 1) + (long)x * (ny + 1) + (z + 1) * sqx] = oX;
    qy[y + (long)(x + 1) * ny + (z + 1) * sqy] = oY;
    qz[(y + 1) + (long)(x + 1) * (ny + 1) + z * sqz] = oZ;
    // entries of q no main write reaches (an index 0 on a potential-staggered axis)
    if (y == 0) {
        qx[(long)x * (ny + 1) + (z + 1) * sqx] = 0.f;
        qz[(long)(x + 1) * (ny + 1) + z * sqz] = 0.f;
    }
    if (z == 0) {
        qx[(y + 1) + (long)x * (ny + 1)] = 0.f;
        qy[y + (long)(x + 1) * ny] = 0.f;
    }
    if (x == 0) {
        qy[y + (z + 1) * sqy] = 0.f;
        qz[(y + 1) + z * sqz] = 0.f;
    }
    if (y == 0 && z == 0) qx[(long)x * (ny + 1)] = 0.f;
    if (x == 0 && z == 0) qy[y] = 0.f;
    if (x == 0 && y == 0) qz[z * sqz] = 0.f;
}

// PZ z-planes per thread, their nine velocity loads issued before any arithmetic (one plane per thread
// left the pass latency bound at ~0.6 of HBM)
constexpr int PZ = 4;
__global__ void __launch_bounds__(256) project3d_kernel(float* __restrict__ qx, float* __restrict__ qy,
                                                        float* __restrict__ qz, const float* __restrict__ xv,
                                                        const float* __restrict__ yv, const float* __restrict__ zv,
                                                        int nx, int ny, int nz, AxisTab tx, AxisTab ty, AxisTab tz) {
    const int y = blockIdx.x * 32 + threadIdx.x;
    const int x = blockIdx.y * 8 + threadIdx.y;
    const int z0 = blockIdx.z * PZ;
    if (y >= ny || x >= nx) return;
    const long sxv = (long)(nx + 1) * ny, syv = (long)nx * (ny + 1), szv = (long)nx * ny;
    float xin[PZ], yin[PZ], zin[PZ];
#pragma unroll
    for (int j = 0; j < PZ; ++j) {
        const int z = z0 + j;
        if (z < nz) {
            xin[j] = xv[y + (long)(x + 1) * ny + z * sxv];
            yin[j] = yv[(y + 1) + (long)x * (ny + 1) + z * syv];
            zin[j] = zv[y + (long)x * ny + (z + 1) * szv];
        }
    }
#pragma unroll
    for (int j = 0; j < PZ; ++j)
        if (z0 + j < nz) project3d_cell(qx, qy, qz, nx, ny, x, y, z0 + j, xin[j], yin[j], zin[j], tx, ty, tz);
}

// The projection with Dirichlet domain walls (the recovery's bc 'd'; cuProjectLocal_q_3d_nq_ccc,
// cuDivLocalProject3D.cu:4474-4877).  Coefficient (x, y, z) as in project3d_kernel; with one index 0 the
// wall-side velocity coefficients X0 = xv(x, y, z), Y0 = yv(x, y, z), Z0 = zv(x, y, z) enter too:
//  * interior: q = (s x v) / |s|^2;
//  * wall plane a = 0: the wall-normal pair (e.g. Z0, Z for z = 0) divided by the scale of the other
//    in-plane axis gives the two potential entries along the wall, their difference times
//    l_a = dx_inv_a / n_a corrects the in-plane velocity, and the remaining component is the
//    one-component ratio weighted by the inner-product tables;
//  * wall line (two indices 0): two such divided pairs, the third component 0;
//  * corner: the wall velocities divided by l.
// Every potential entry with an index 0 along one of its own axes is written by exactly one thread
// (zeros included), so q needs no clearing.
__global__ void __launch_bounds__(256) project3d_nq_kernel(float* __restrict__ qx, float* __restrict__ qy,
                                                           float* __restrict__ qz, const float* __restrict__ xv,
                                                           const float* __restrict__ yv, const float* __restrict__ zv,
                                                           int nx, int ny, int nz, AxisTab tx, AxisTab ty, AxisTab tz,
                                                           float lx, float ly, float lz) {
    const int y = blockIdx.x * 32 + threadIdx.x;
    const int x = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (y >= ny || x >= nx) return;
    const long sxv = (long)(nx + 1) * ny, syv = (long)nx * (ny + 1), szv = (long)nx * ny;
    const long pqx = (long)nx * (ny + 1), pqy = (long)(nx + 1) * ny, pqz = (long)(nx + 1) * (ny + 1);
    auto QX = [&](int i, int j, int k) -> float& { return qx[j + (long)i * (ny + 1) + k * pqx]; };
    auto QY = [&](int i, int j, int k) -> float& { return qy[j + (long)i * ny + k * pqy]; };
    auto QZ = [&](int i, int j, int k) -> float& { return qz[j + (long)i * (ny + 1) + k * pqz]; };
    float X = xv[y + (long)(x + 1) * ny + z * sxv];
    float Y = yv[(y + 1) + (long)x * (ny + 1) + z * syv];
    float Z = zv[y + (long)x * ny + (z + 1) * szv];
    const float sx = tx.s[x], sy = ty.s[y], sz = tz.s[z];
    float oX = 0.f, oY = 0.f, oZ = 0.f;
    const bool ix = x == 0, iy = y == 0, iz = z == 0;
    if (!ix && !iy && !iz) {
        const float inv = 1.f / (sy * sy + sx * sx + sz * sz);
        oZ = (sy * X - sx * Y) * inv;
        oX = (sz * Y - sy * Z) * inv;
        oY = (sx * Z - sz * X) * inv;
    } else {
        const float ip0x = tx.ip0[x], ip1x = tx.ip1[x], ip0y = ty.ip0[y], ip1y = ty.ip1[y];
        const float ip0z = tz.ip0[z], ip1z = tz.ip1[z];
        const float b010 = ip0x * ip1y * ip0z, b100 = ip1x * ip0y * ip0z, b001 = ip0x * ip0y * ip1z;
        const float X0 = ix ? xv[y + z * sxv] : 0.f;
        const float Y0 = iy ? yv[(long)x * (ny + 1) + z * syv] : 0.f;
        const float Z0 = iz ? zv[y + (long)x * ny] : 0.f;
        if (iz && !ix && !iy) {  // wall plane z = 0
            const float t0 = Z0 / sx, t1 = Z / sx;
            X += (t1 - t0) * lz;
            QX(x, y + 1, 0) = 0.f;
            QY(x + 1, y, 0) = t0;
            oY = t1;
            oZ = (X * (sy * b100) - Y * (sx * b010)) * (1.f / (sx * (sx * b010) + sy * (sy * b100) + kEps));
        } else if (iy && !ix && !iz) {  // wall plane y = 0
            const float t0 = Y0 / sz, t1 = Y / sz;
            Z += (t1 - t0) * ly;
            QX(x, 0, z + 1) = t0;
            QZ(x + 1, 0, z) = 0.f;
            oX = t1;
            oY = (Z * (sx * b001) - X * (sz * b100)) * (1.f / (sx * (sx * b001) + sz * (sz * b100) + kEps));
        } else if (ix && !iy && !iz) {  // wall plane x = 0
            const float t0 = X0 / sy, t1 = X / sy;
            Y += (t1 - t0) * lx;
            QZ(0, y + 1, z) = t0;
            QY(0, y, z + 1) = 0.f;
            oZ = t1;
            oX = (Y * (sz * b010) - Z * (sy * b001)) * (1.f / (sy * (sy * b001) + sz * (sz * b010) + kEps));
        } else if (!ix && iy && iz) {  // wall line along x
            QY(x + 1, 0, 0) = Z0 / sx;
            QZ(x + 1, 0, 0) = -Y0 / sx;
            QX(x, 0, 1) = 0.f;
            QX(x, 0, 0) = 0.f;
            QX(x, 1, 0) = 0.f;
            oY = Z / sx;
            oZ = -Y / sx;
        } else if (ix && !iy && iz) {  // wall line along y
            QX(0, y + 1, 0) = -Z0 / sy;
            QZ(0, y + 1, 0) = X0 / sy;
            QY(0, y, 0) = 0.f;
            QY(1, y, 0) = 0.f;
            QY(0, y, 1) = 0.f;
            oX = -Z / sy;
            oZ = X / sy;
        } else if (ix && iy && !iz) {  // wall line along z
            QX(0, 0, z + 1) = Y0 / sz;
            QY(0, 0, z + 1) = -X0 / sz;
            QZ(0, 0, z) = 0.f;
            QZ(0, 1, z) = 0.f;
            QZ(1, 0, z) = 0.f;
            oX = Y / sz;
            oY = -X / sz;
        } else {  // corner
            const float x010 = -Z0 / ly;
            QZ(0, 0, 0) = 0.f;
            QZ(1, 0, 0) = 0.f;
            QZ(0, 1, 0) = 0.f;
            QX(0, 0, 0) = 0.f;
            QX(0, 1, 0) = x010;
            QX(0, 0, 1) = Y0 / lz;
            QY(0, 0, 0) = 0.f;
            QY(1, 0, 0) = 0.f;
            QY(0, 0, 1) = -X0 / lz;
            oX = x010 + Y / lz;
            oY = -X / lz;
        }
    }
    QX(x, y + 1, z + 1) = oX;
    QY(x + 1, y, z + 1) = oY;
    QZ(x + 1, y + 1, z) = oZ;
}

__global__ void __launch_bounds__(256) project2d_kernel(float* __restrict__ qz, const float* __restrict__ xv,
                                                        const float* __restrict__ yv, int nx, int ny, AxisTab tx,
                                                        AxisTab ty) {
    const int y = blockIdx.x * 32 + threadIdx.x;  // qz index along y in [0, ny]
    const int x = blockIdx.y * 8 + threadIdx.y;   // qz index along x in [0, nx]
    if (y > ny || x > nx) return;
    float out = 0.f;
    if (x >= 2 && y >= 2) {
        const int i = x - 1, j = y - 1;
        const float sx = tx.s[i], sy = ty.s[j];
        const float ip0x = tx.ip0[i], ip1x = tx.ip1[i], ip0y = ty.ip0[j], ip1y = ty.ip1[j];
        const float xin = xv[j + (long)x * ny];
        const float yin = yv[y + (long)i * (ny + 1)];
        const float mid = sx * sx * ip0x * ip1y + sy * sy * ip1x * ip0y + kEps;
        out = (xin * sy * ip1x * ip0y - yin * sx * ip0x * ip1y) / mid;
    }
    qz[y + (long)x * (ny + 1)] = out;
}

// What the 2D Dirichlet-wall projection reads besides the axis tables: per axis the base table's
// entries (0, 0) and (0, 1) and the wall scale dx_inv / n, and the corner map of GetDivL0Matrix.
struct Edge2D {
    float b00[2], b01[2], se[2];
    float l0[16];
};

// cuProjectLocal_q_single_n (cuDivLocalProject.cu:1047-1460), the projection of a 2D recovery with
// Dirichlet walls, one thread per qz entry (x, y) in [0, nx] x [0, ny] with X(x, y) = xv(x, y - 1),
// Y(x, y) = yv(x - 1, y) (0 outside): the pointwise ratio for x, y >= 2 (half from each of the
// reference's two passes); at x in {0, 1} (y >= 2) the pass along y solves a 2 x 2 system that couples
// X(0, y), X(1, y) and Y(1, y); at y in {0, 1} (x >= 2) the pass along x the same with the axes
// swapped; the four corner entries are the GetDivL0Matrix map of X(0, 1), X(1, 1), Y(1, 0), Y(1, 1).
__global__ void __launch_bounds__(256) project2d_nq_kernel(float* __restrict__ qz, const float* __restrict__ xv,
                                                           const float* __restrict__ yv, int nx, int ny, AxisTab tx,
                                                           AxisTab ty, Edge2D e) {
    const int y = blockIdx.x * 32 + threadIdx.x;
    const int x = blockIdx.y * 8 + threadIdx.y;
    if (y > ny || x > nx) return;
    auto X = [&](int a, int b) { return b > 0 ? xv[(b - 1) + (long)a * ny] : 0.f; };
    auto Y = [&](int a, int b) { return a > 0 ? yv[b + (long)(a - 1) * (ny + 1)] : 0.f; };
    const float sx = tx.s[x > 0 ? x - 1 : 0], sy = ty.s[y > 0 ? y - 1 : 0];
    float qx = 0.f, qy = 0.f;
    if (x >= 2 && y >= 2) {
        const float ip0x = tx.ip0[x - 1], ip1x = tx.ip1[x - 1], ip0y = ty.ip0[y - 1], ip1y = ty.ip1[y - 1];
        const float xin = X(x, y), yin = Y(x, y);
        const float m1 = sx * sx * ip0x * ip1y + sy * sy * ip1x * ip0y + kEps;
        qy = 0.5f * ((xin * sy * ip1x * ip0y - yin * sx * ip0x * ip1y) / m1);
        const float m2 = sy * sy * ip0y * ip1x + sx * sx * ip1y * ip0x + kEps;
        qx = 0.5f * ((xin * sy * ip0y * ip1x - yin * sx * ip1y * ip0x) / m2);
    } else if (y >= 2) {
        const float se = e.se[0], ip0x = tx.ip0[0], b00 = e.b00[0], b01 = e.b01[0];
        const float ip0y = ty.ip0[y - 1], ip1y = ty.ip1[y - 1];
        const float ye = Y(1, y), x0 = X(0, y), x1 = X(1, y);
        float m0 = se * se * ip0x * ip1y + sy * sy * b00 * ip0y;
        float m1 = -se * se * ip0x * ip1y + sy * sy * b01 * ip0y;
        const float dv = m0 * m0 - m1 * m1 + kEps;
        m0 /= dv;
        m1 /= -dv;
        float f1 = ye * se * ip0x * ip1y;
        f1 += x0 * sy * b00 * ip0y;
        f1 += x1 * sy * b01 * ip0y;
        float f2 = -ye * se * ip0x * ip1y;
        f2 += x0 * sy * b01 * ip0y;
        f2 += x1 * sy * b00 * ip0y;
        qy = x == 0 ? m0 * f1 + m1 * f2 : m1 * f1 + m0 * f2;
    } else if (x >= 2) {
        const float se = e.se[1], ip0y = ty.ip0[0], b00 = e.b00[1], b01 = e.b01[1];
        const float ip0x = tx.ip0[x - 1], ip1x = tx.ip1[x - 1];
        const float xe = X(x, 1), y0 = Y(x, 0), y1 = Y(x, 1);
        float m0 = sx * sx * ip0x * b00 + se * se * ip1x * ip0y;
        float m1 = sx * sx * ip0x * b01 - se * se * ip1x * ip0y;
        const float dv = m0 * m0 - m1 * m1 + kEps;
        m0 /= dv;
        m1 /= -dv;
        const float a00 = ip0x * b00, a01 = ip0x * b01;
        float f1 = -xe * se * ip1x * ip0y;
        f1 -= y0 * sx * a00;
        f1 -= y1 * sx * a01;
        float f2 = xe * se * ip1x * ip0y;
        f2 -= y0 * sx * a01;
        f2 -= y1 * sx * a00;
        qx = y == 0 ? m0 * f1 + m1 * f2 : m1 * f1 + m0 * f2;
    } else {
        const float* a = e.l0 + 4 * (2 * y + x);
        qx = a[2] * X(0, 1) + a[3] * X(1, 1) - a[0] * Y(1, 0) - a[1] * Y(1, 1);
    }
    qz[y + (long)x * (ny + 1)] = qx + qy;
}

// GetDivL0Matrix (DivL0Matrix.cpp:3-46), by the difference of the two axes' levels; the reference's
// entry for a difference of 5 has minus signs where the others have commas, so its first value is the
// sum of the four numbers and the rest are 0, evaluated here the same way.
void div_l0_matrix(float* dst, int lx, int ly) {
    const int m = std::min(lx, ly), mx = lx - m, my = ly - m, k = std::max(mx, my);
    static const double T[8][4] = {
        {-0.600000000000000, -0.400000000000000, -0.450000000000000, -0.050000000000000},
        {-1.058823529411764, -0.941176470588235, -0.485294117647059, -0.014705882352941},
        {-2.030769230769231, -1.969230769230771, -0.496153846153847, -0.003846153846153},
        {-4.015564202334636, -3.984435797665360, -0.499027237354084, -0.000972762645915},
        {0, 0, 0, 0},
        {-16.003905296558496, -15.996094703441514, -0.499938979741274, -0.000061020258726},
        {-32.001953005797915, -31.998046994202070, -0.499984742142203, -0.000015257857796},
        {-64.000976547601056, -63.999023452398980, -0.499996185360941, -0.000003814639067}};
    double r[4] = {-0.374999999999990, -0.124999999999991, -0.375000000000009, -0.125000000000009};
    if (k == 5) {
        r[0] = -8.007804878048813 - 7.992195121951190 - 0.499756097560973 - 0.000243902439025;
        r[1] = r[2] = r[3] = 0.0;
    } else if (k >= 1 && k <= 8) {
        for (int i = 0; i < 4; ++i) r[i] = T[k - 1][i];
    }
    if (mx < my) {
        std::swap(r[0], r[2]);
        std::swap(r[1], r[3]);
    }
    const double v[16] = {r[0], r[1], r[2], r[3], -r[0], -r[1], r[3], r[2],
                          r[1], r[0], -r[2], -r[3], -r[1], -r[0], -r[3], -r[2]};
    for (int i = 0; i < 16; ++i) dst[i] = (float)v[i];
}

// Builds the per-axis table [s | ip0 | ip1] (length 3n floats) on the device.  wall: the walls'
// boundary type; the projection wavelet CDF3.7 takes it, the base wavelet CDF4.6 the other one
// (CuDivLocalProject3D's constructor, cuDivLocalProject3D.cu:50-60, with bc = proj_bc(wall)).
// edge (when not null): the base table's entries (0, 0) and (0, 1), which the 2D Dirichlet-wall
// projection reads at its walls.
wp_status build_axis_table(float** d_tab, int n, double h, cudaStream_t s, char wall = 'n', float* edge = nullptr) {
    const int L = wp_ilog2(n);
    double* d_ip = nullptr;
    WP_CUDA_TRY(cudaMalloc((void**)&d_ip, sizeof(double) * (2 * n + 2)));
    wp_status st = wp_ip_diag_device(d_ip, n, WP_ID_CDF3_7, wall, s);
    if (st == WP_OK) st = wp_ip_diag_device(d_ip + n, n + 1, WP_ID_CDF4_6, wall == 'n' ? 'd' : 'n', s);
    if (st == WP_OK && edge) st = wp_ip_gram01_device(d_ip + 2 * n + 1, n + 1, WP_ID_CDF4_6, wall == 'n' ? 'd' : 'n', s);
    std::vector<double> ip(2 * n + 2);
    if (st == WP_OK) {
        cudaError_t e = cudaMemcpyAsync(ip.data(), d_ip, sizeof(double) * (2 * n + 2), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { wp_set_cuda_error(e, "ip table copy", __FILE__, __LINE__); st = WP_ERR_CUDA; }
    }
    cudaFree(d_ip);
    if (st != WP_OK) return st;
    std::vector<float> tab(3 * n);
    for (int i = 0; i < n; ++i) {
        int bl = 0;
        for (int v = i; v > 0; v >>= 1) ++bl;
        const int j = L - bl + 1;
        tab[i] = (float)(4.0 / h / ((double)(1 << j) + 1e-12));
        tab[n + i] = (float)ip[i];              // ip_proj[i]  (CDF3.7, n points)
        tab[2 * n + i] = (float)ip[n + i + 1];  // ip_base[i+1] (CDF4.6, n+1 points)
    }
    if (edge) {
        edge[0] = (float)ip[n];          // ip_base[0]
        edge[1] = (float)ip[2 * n + 1];  // Gram entry (0, 1) of the base wavelet
    }
    WP_CUDA_TRY(cudaMalloc((void**)d_tab, sizeof(float) * 3 * n));
    WP_CUDA_TRY(cudaMemcpy(*d_tab, tab.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice));
    return WP_OK;
}

AxisTab view(const float* t, int n) { return AxisTab{t, t + n, t + 2 * n}; }

bool check_wavelets(int curl, int div) { return curl == WP_ID_CDF3_7 && div == WP_ID_CDF4_6; }

}  // namespace

struct wp_recover3d {
    int n[3];
    int L[3];
    double h[3];
    char bc, bcd;  // the walls' boundary type and the div wavelet's (the other one)
    float* tab[3];
    float* tmp[3];
};

extern "C" CUWHHD_API wp_status wp_recover3d_create(wp_recover3d** out, int nx, int ny, int nz, double dx, double dy,
                                                    double dz, char bc, int curl_wavelet, int div_wavelet) {
    if (!out) { wp_set_error_msg("wp_recover3d_create: null handle"); return WP_ERR_INVALID_ARG; }
    *out = nullptr;
    if (!wp_is_pow2(nx) || !wp_is_pow2(ny) || !wp_is_pow2(nz) || nx < 4 || ny < 4 || nz < 4 || nx > 4096 ||
        ny > 4096 || nz > 4096 || !(dx > 0) || !(dy > 0) || !(dz > 0)) {
        wp_set_error_msg("wp_recover3d_create: extents must be powers of two in [4, 4096] and spacings > 0");
        return WP_ERR_INVALID_ARG;
    }
    if (bc != 'n' && bc != 'd') { wp_set_error_msg("wp_recover3d_create: bc must be 'n' (zero-normal-flux walls) or 'd' (Dirichlet walls)"); return WP_ERR_UNSUPPORTED; }
    if (!check_wavelets(curl_wavelet, div_wavelet)) { wp_set_error_msg("wp_recover3d_create: curl CDF3.7 / div CDF4.6 only"); return WP_ERR_UNSUPPORTED; }
    wp_recover3d* h = new (std::nothrow) wp_recover3d();
    if (!h) return WP_ERR_INVALID_ARG;
    h->bc = bc;
    h->bcd = bc == 'n' ? 'd' : 'n';
    int n[3] = {nx, ny, nz};
    double hs[3] = {dx, dy, dz};
    for (int a = 0; a < 3; ++a) {
        h->n[a] = n[a];
        h->L[a] = wp_ilog2(n[a]);
        h->h[a] = hs[a];
        wp_status st = build_axis_table(&h->tab[a], n[a], hs[a], 0, bc);
        if (st != WP_OK) { wp_recover3d_destroy(h); return st; }
    }
    if (cudaError_t e = wp_dwt_prepare(); e != cudaSuccess) {
        wp_set_cuda_error(e, "recover3d filters", __FILE__, __LINE__);
        wp_recover3d_destroy(h);
        return WP_ERR_CUDA;
    }
    size_t sz[3] = {(size_t)(nx + 1) * ny * nz, (size_t)nx * (ny + 1) * nz, (size_t)nx * ny * (nz + 1)};
    for (int a = 0; a < 3; ++a) {
        cudaError_t e = cudaMalloc((void**)&h->tmp[a], sizeof(float) * sz[a]);
        if (e != cudaSuccess) { wp_set_cuda_error(e, "recover3d temp", __FILE__, __LINE__); wp_recover3d_destroy(h); return WP_ERR_CUDA; }
    }
    // tile widths of the 18 passes, measured once per shape for the process (on a scratch array
    // as large as the largest potential component)
    {
        float* scratch = nullptr;
        const size_t big = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
        if (cudaMalloc((void**)&scratch, sizeof(float) * big) == cudaSuccess) {
            cudaMemset(scratch, 0, sizeof(float) * big);
            const int C = WP_ID_CDF3_7, V = WP_ID_CDF4_6;
            const int Lx = h->L[0], Ly = h->L[1], Lz = h->L[2];
            const char b = h->bc, d = h->bcd;
            struct P { int dx, dy, dz, L; char ax; int w; char bc; int f; };
            const P passes[18] = {
                {nx + 1, ny, nz, Lx, 'x', V, d, 1}, {nx + 1, ny, nz, Ly, 'y', C, b, 1}, {nx + 1, ny, nz, Lz, 'z', C, b, 1},
                {nx, ny + 1, nz, Lx, 'x', C, b, 1}, {nx, ny + 1, nz, Ly, 'y', V, d, 1}, {nx, ny + 1, nz, Lz, 'z', C, b, 1},
                {nx, ny, nz + 1, Lx, 'x', C, b, 1}, {nx, ny, nz + 1, Ly, 'y', C, b, 1}, {nx, ny, nz + 1, Lz, 'z', V, d, 1},
                {nx, ny + 1, nz + 1, Lx, 'x', C, b, 0}, {nx, ny + 1, nz + 1, Ly, 'y', V, d, 0}, {nx, ny + 1, nz + 1, Lz, 'z', V, d, 0},
                {nx + 1, ny, nz + 1, Lx, 'x', V, d, 0}, {nx + 1, ny, nz + 1, Ly, 'y', C, b, 0}, {nx + 1, ny, nz + 1, Lz, 'z', V, d, 0},
                {nx + 1, ny + 1, nz, Lx, 'x', V, d, 0}, {nx + 1, ny + 1, nz, Ly, 'y', V, d, 0}, {nx + 1, ny + 1, nz, Lz, 'z', C, b, 0}};
            for (const P& q : passes)
                if (wp_dwt_axis_tune<float>(scratch, q.dx, q.dy, q.dz, q.L, q.ax, q.w, q.bc, q.f, nullptr) != WP_OK) break;
            cudaDeviceSynchronize();
            cudaFree(scratch);
        } else {
            cudaGetLastError();
        }
    }
    *out = h;
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_recover3d_destroy(wp_recover3d* h) {
    if (!h) return WP_OK;
    for (int a = 0; a < 3; ++a) {
        if (h->tab[a]) cudaFree(h->tab[a]);
        if (h->tmp[a]) cudaFree(h->tmp[a]);
    }
    delete h;
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_recover3d_project(wp_recover3d* h, float* qx, float* qy, float* qz,
                                                     const float* xv, const float* yv, const float* zv, void* stream) {
    if (!h || !qx || !qy || !qz || !xv || !yv || !zv) { wp_set_error_msg("wp_recover3d_project: null pointer"); return WP_ERR_INVALID_ARG; }
    const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
    if (nz > 65535) return WP_ERR_UNSUPPORTED;
    dim3 grid(wp_cdiv(ny, 32), wp_cdiv(nx, 8), nz);
    cudaStream_t s = (cudaStream_t)stream;
    const double bytes = 4.0 * ((double)(nx + 1) * ny * nz * 3 + (double)(nx + 1) * (ny + 1) * nz * 3);
    if (h->bc == 'd') {
        // the reference's l = dx_inv / n, formed in FP32 as its FP32 build does
        const float lx = (1.f / (float)h->h[0]) / (float)nx, ly = (1.f / (float)h->h[1]) / (float)ny;
        const float lz = (1.f / (float)h->h[2]) / (float)nz;
        WP_KERNEL("project3d", bytes, s,
                  project3d_nq_kernel<<<grid, dim3(32, 8), 0, s>>>(qx, qy, qz, xv, yv, zv, nx, ny, nz,
                                                                   view(h->tab[0], nx), view(h->tab[1], ny),
                                                                   view(h->tab[2], nz), lx, ly, lz));
        return WP_OK;
    }
    const dim3 gridp(wp_cdiv(ny, 32), wp_cdiv(nx, 8), wp_cdiv(nz, PZ));
    WP_KERNEL("project3d", bytes, s,
              project3d_kernel<<<gridp, dim3(32, 8), 0, s>>>(qx, qy, qz, xv, yv, zv, nx, ny, nz, view(h->tab[0], nx),
                                                             view(h->tab[1], ny), view(h->tab[2], nz)));
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_recover3d_run(wp_recover3d* h, float* qx, float* qy, float* qz, const float* xv,
                                                 const float* yv, const float* zv, void* stream) {
    if (!h || !qx || !qy || !qz || !xv || !yv || !zv) { wp_set_error_msg("wp_recover3d_run: null pointer"); return WP_ERR_INVALID_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
    const int Lx = h->L[0], Ly = h->L[1], Lz = h->L[2];
    const int C = WP_ID_CDF3_7, V = WP_ID_CDF4_6;
    float *tx = h->tmp[0], *ty = h->tmp[1], *tz = h->tmp[2];
    const char b = h->bc, d = h->bcd;  // curl wavelet: the walls' type; div wavelet: the other
    wp_status st;
#define WP_T(dst, src, DX, DY, DZ, L, ax, w, bc, f)                                          \
    if ((st = wp_dwt_axis_launch<float>(dst, src, DX, DY, DZ, L, ax, w, bc, f, s)) != WP_OK) \
        return st;
    // forward analysis (cuWaveletPotentialRecover3D.cu:32-42)
    WP_T(tx, xv, nx + 1, ny, nz, Lx, 'x', V, d, 1);
    WP_T(tx, tx, nx + 1, ny, nz, Ly, 'y', C, b, 1);
    WP_T(tx, tx, nx + 1, ny, nz, Lz, 'z', C, b, 1);
    WP_T(ty, yv, nx, ny + 1, nz, Lx, 'x', C, b, 1);
    WP_T(ty, ty, nx, ny + 1, nz, Ly, 'y', V, d, 1);
    WP_T(ty, ty, nx, ny + 1, nz, Lz, 'z', C, b, 1);
    WP_T(tz, zv, nx, ny, nz + 1, Lx, 'x', C, b, 1);
    WP_T(tz, tz, nx, ny, nz + 1, Ly, 'y', C, b, 1);
    WP_T(tz, tz, nx, ny, nz + 1, Lz, 'z', V, d, 1);
    // local projection (:46)
    if ((st = wp_recover3d_project(h, qx, qy, qz, tx, ty, tz, stream)) != WP_OK) return st;
    // inverse synthesis (:50-60)
    WP_T(qx, qx, nx, ny + 1, nz + 1, Lx, 'x', C, b, 0);
    WP_T(qx, qx, nx, ny + 1, nz + 1, Ly, 'y', V, d, 0);
    WP_T(qx, qx, nx, ny + 1, nz + 1, Lz, 'z', V, d, 0);
    WP_T(qy, qy, nx + 1, ny, nz + 1, Lx, 'x', V, d, 0);
    WP_T(qy, qy, nx + 1, ny, nz + 1, Ly, 'y', C, b, 0);
    WP_T(qy, qy, nx + 1, ny, nz + 1, Lz, 'z', V, d, 0);
    WP_T(qz, qz, nx + 1, ny + 1, nz, Lx, 'x', V, d, 0);
    WP_T(qz, qz, nx + 1, ny + 1, nz, Ly, 'y', V, d, 0);
    WP_T(qz, qz, nx + 1, ny + 1, nz, Lz, 'z', C, b, 0);
#undef WP_T
    return WP_OK;
}

// CuWaveletPotentialRecover3D::CutCoefficients (cuWaveletPotentialRecover3D.cu:123-239): in the
// analysed potential, every cell (x, y, z) of the (nx+1, ny+1, nz+1) index box whose coefficient
// level along some axis a, j_a = L_a - bitlength(max(i_a - 1, 0)), is below `cut` clears the three
// components there: qx at (x-1, y, z), qy at (x, y-1, z), qz at (x, y, z-1), each where its index
// exists (the reference's cuCutCoefs, with the same guards).
__global__ void cut_coefs_kernel(float* __restrict__ qx, float* __restrict__ qy, float* __restrict__ qz, int nx,
                                 int ny, int nz, int Lx, int Ly, int Lz, int cut) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y, z = blockIdx.z;
    if (y > ny) return;
    const int jx = Lx - (32 - __clz(max(x - 1, 0)));
    const int jy = Ly - (32 - __clz(max(y - 1, 0)));
    const int jz = Lz - (32 - __clz(max(z - 1, 0)));
    if (jx >= cut && jy >= cut && jz >= cut) return;
    // with cut <= min(L) a level below the cut needs an index >= 2 along that axis, so the
    // component shifted along it exists; the other two are guarded as in the reference
    if (x > 0 || jx < cut) qx[y + (long)(x - 1) * (ny + 1) + (long)z * nx * (ny + 1)] = 0.f;
    if (y > 0 || jy < cut) qy[(y - 1) + (long)x * ny + (long)z * (nx + 1) * ny] = 0.f;
    if (z > 0 || jz < cut) qz[y + (long)x * (ny + 1) + (long)(z - 1) * (nx + 1) * (ny + 1)] = 0.f;
}

extern "C" CUWHHD_API wp_status wp_recover3d_cut(wp_recover3d* h, float* qx_out, float* qy_out, float* qz_out,
                                                 const float* qx, const float* qy, const float* qz, int level,
                                                 void* stream) {
    if (!h || !qx_out || !qy_out || !qz_out || !qx || !qy || !qz) {
        wp_set_error_msg("wp_recover3d_cut: null pointer");
        return WP_ERR_INVALID_ARG;
    }
    if (h->bc != 'n') {
        wp_set_error_msg("wp_recover3d_cut: only handles with bc 'n' (zero-normal-flux walls)");
        return WP_ERR_UNSUPPORTED;
    }
    const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
    const int Lx = h->L[0], Ly = h->L[1], Lz = h->L[2];
    if (level < 0 || level > std::min(Lx, std::min(Ly, Lz))) {
        wp_set_error_msg("wp_recover3d_cut: level must lie in [0, min(levels)]");
        return WP_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int C = WP_ID_CDF3_7, V = WP_ID_CDF4_6;
    wp_status st;
#define WP_T(dst, src, DX, DY, DZ, L, ax, w, bc, f)                                          \
    if ((st = wp_dwt_axis_launch<float>(dst, src, DX, DY, DZ, L, ax, w, bc, f, s)) != WP_OK) \
        return st;
    // analysis of each component with the recovery's synthesis wavelets (:205-215)
    WP_T(qx_out, qx, nx, ny + 1, nz + 1, Lx, 'x', C, 'n', 1);
    WP_T(qx_out, qx_out, nx, ny + 1, nz + 1, Ly, 'y', V, 'd', 1);
    WP_T(qx_out, qx_out, nx, ny + 1, nz + 1, Lz, 'z', V, 'd', 1);
    WP_T(qy_out, qy, nx + 1, ny, nz + 1, Lx, 'x', V, 'd', 1);
    WP_T(qy_out, qy_out, nx + 1, ny, nz + 1, Ly, 'y', C, 'n', 1);
    WP_T(qy_out, qy_out, nx + 1, ny, nz + 1, Lz, 'z', V, 'd', 1);
    WP_T(qz_out, qz, nx + 1, ny + 1, nz, Lx, 'x', V, 'd', 1);
    WP_T(qz_out, qz_out, nx + 1, ny + 1, nz, Ly, 'y', V, 'd', 1);
    WP_T(qz_out, qz_out, nx + 1, ny + 1, nz, Lz, 'z', C, 'n', 1);
    // the cut (:221-222)
    const dim3 g((unsigned)wp_cdiv(ny + 1, 128), nx + 1, nz + 1);
    const double bytes = 4.0 * 3.0 * (double)(nx + 1) * (ny + 1) * (nz + 1);
    WP_KERNEL("cut_coefs", bytes, s,
              cut_coefs_kernel<<<g, 128, 0, s>>>(qx_out, qy_out, qz_out, nx, ny, nz, Lx, Ly, Lz, level));
    // synthesis (:228-238)
    WP_T(qx_out, qx_out, nx, ny + 1, nz + 1, Lx, 'x', C, 'n', 0);
    WP_T(qx_out, qx_out, nx, ny + 1, nz + 1, Ly, 'y', V, 'd', 0);
    WP_T(qx_out, qx_out, nx, ny + 1, nz + 1, Lz, 'z', V, 'd', 0);
    WP_T(qy_out, qy_out, nx + 1, ny, nz + 1, Lx, 'x', V, 'd', 0);
    WP_T(qy_out, qy_out, nx + 1, ny, nz + 1, Ly, 'y', C, 'n', 0);
    WP_T(qy_out, qy_out, nx + 1, ny, nz + 1, Lz, 'z', V, 'd', 0);
    WP_T(qz_out, qz_out, nx + 1, ny + 1, nz, Lx, 'x', V, 'd', 0);
    WP_T(qz_out, qz_out, nx + 1, ny + 1, nz, Ly, 'y', V, 'd', 0);
    WP_T(qz_out, qz_out, nx + 1, ny + 1, nz, Lz, 'z', C, 'n', 0);
#undef WP_T
    return WP_OK;
}

struct wp_recover2d {
    int n[2];
    int L[2];
    double h[2];
    char bc, bcd;  // the walls' boundary type and the div wavelet's (the other one)
    Edge2D edge;   // bc 'd': what the projection reads at the walls
    float* tab[2];
    float* tmp[2];
};

extern "C" CUWHHD_API wp_status wp_recover2d_create(wp_recover2d** out, int nx, int ny, double dx, double dy, char bc,
                                                    int curl_wavelet, int div_wavelet) {
    if (!out) { wp_set_error_msg("wp_recover2d_create: null handle"); return WP_ERR_INVALID_ARG; }
    *out = nullptr;
    if (!wp_is_pow2(nx) || !wp_is_pow2(ny) || nx < 4 || ny < 4 || nx > 4096 || ny > 4096 || !(dx > 0) || !(dy > 0)) {
        wp_set_error_msg("wp_recover2d_create: extents must be powers of two in [4, 4096] and spacings > 0");
        return WP_ERR_INVALID_ARG;
    }
    if (bc != 'n' && bc != 'd') {
        wp_set_error_msg("wp_recover2d_create: bc must be 'n' (zero-normal-flux walls) or 'd' (Dirichlet walls)");
        return WP_ERR_UNSUPPORTED;
    }
    if (!check_wavelets(curl_wavelet, div_wavelet)) { wp_set_error_msg("wp_recover2d_create: curl CDF3.7 / div CDF4.6 only"); return WP_ERR_UNSUPPORTED; }
    wp_recover2d* h = new (std::nothrow) wp_recover2d();
    if (!h) return WP_ERR_INVALID_ARG;
    h->bc = bc;
    h->bcd = bc == 'n' ? 'd' : 'n';
    int n[2] = {nx, ny};
    double hs[2] = {dx, dy};
    for (int a = 0; a < 2; ++a) {
        h->n[a] = n[a];
        h->L[a] = wp_ilog2(n[a]);
        h->h[a] = hs[a];
        float edge[2] = {0.f, 0.f};
        wp_status st = build_axis_table(&h->tab[a], n[a], hs[a], 0, bc, bc == 'd' ? edge : nullptr);
        if (st != WP_OK) { wp_recover2d_destroy(h); return st; }
        h->edge.b00[a] = edge[0];
        h->edge.b01[a] = edge[1];
        h->edge.se[a] = (float)(1.0 / hs[a] / n[a]);
    }
    div_l0_matrix(h->edge.l0, h->L[0], h->L[1]);
    if (cudaError_t e = wp_dwt_prepare(); e != cudaSuccess) {
        wp_set_cuda_error(e, "recover2d filters", __FILE__, __LINE__);
        wp_recover2d_destroy(h);
        return WP_ERR_CUDA;
    }
    size_t sz[2] = {(size_t)(nx + 1) * ny, (size_t)nx * (ny + 1)};
    for (int a = 0; a < 2; ++a) {
        cudaError_t e = cudaMalloc((void**)&h->tmp[a], sizeof(float) * sz[a]);
        if (e != cudaSuccess) { wp_set_cuda_error(e, "recover2d temp", __FILE__, __LINE__); wp_recover2d_destroy(h); return WP_ERR_CUDA; }
    }
    *out = h;
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_recover2d_destroy(wp_recover2d* h) {
    if (!h) return WP_OK;
    for (int a = 0; a < 2; ++a) {
        if (h->tab[a]) cudaFree(h->tab[a]);
        if (h->tmp[a]) cudaFree(h->tmp[a]);
    }
    delete h;
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_recover2d_project(wp_recover2d* h, float* qz, const float* xv, const float* yv,
                                                     void* stream) {
    if (!h || !qz || !xv || !yv) { wp_set_error_msg("wp_recover2d_project: null pointer"); return WP_ERR_INVALID_ARG; }
    const int nx = h->n[0], ny = h->n[1];
    dim3 grid(wp_cdiv(ny + 1, 32), wp_cdiv(nx + 1, 8));
    cudaStream_t s = (cudaStream_t)stream;
    if (h->bc == 'd') {
        WP_KERNEL("project2d", 4.0 * ((double)(nx + 1) * ny * 2 + (double)(nx + 1) * (ny + 1)), s,
                  project2d_nq_kernel<<<grid, dim3(32, 8), 0, s>>>(qz, xv, yv, nx, ny, view(h->tab[0], nx),
                                                                   view(h->tab[1], ny), h->edge));
        return WP_OK;
    }
    WP_KERNEL("project2d", 4.0 * ((double)(nx + 1) * ny * 2 + (double)(nx + 1) * (ny + 1)), s,
              project2d_kernel<<<grid, dim3(32, 8), 0, s>>>(qz, xv, yv, nx, ny, view(h->tab[0], nx), view(h->tab[1], ny)));
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_recover2d_run(wp_recover2d* h, float* qz, const float* xv, const float* yv,
                                                 void* stream) {
    if (!h || !qz || !xv || !yv) { wp_set_error_msg("wp_recover2d_run: null pointer"); return WP_ERR_INVALID_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    const int nx = h->n[0], ny = h->n[1], Lx = h->L[0], Ly = h->L[1];
    const int C = WP_ID_CDF3_7, V = WP_ID_CDF4_6;
    float *tx = h->tmp[0], *ty = h->tmp[1];
    wp_status st;
    const char b = h->bc, d = h->bcd;
    if ((st = wp_dwt_axis_launch<float>(tx, xv, nx + 1, ny, 1, Lx, 'x', V, d, 1, s)) != WP_OK) return st;
    if ((st = wp_dwt_axis_launch<float>(tx, tx, nx + 1, ny, 1, Ly, 'y', C, b, 1, s)) != WP_OK) return st;
    if ((st = wp_dwt_axis_launch<float>(ty, yv, nx, ny + 1, 1, Lx, 'x', C, b, 1, s)) != WP_OK) return st;
    if ((st = wp_dwt_axis_launch<float>(ty, ty, nx, ny + 1, 1, Ly, 'y', V, d, 1, s)) != WP_OK) return st;
    if ((st = wp_recover2d_project(h, qz, tx, ty, stream)) != WP_OK) return st;
    if ((st = wp_dwt_axis_launch<float>(qz, qz, nx + 1, ny + 1, 1, Lx, 'x', V, d, 0, s)) != WP_OK) return st;
    if ((st = wp_dwt_axis_launch<float>(qz, qz, nx + 1, ny + 1, 1, Ly, 'y', V, d, 0, s)) != WP_OK) return st;
    return WP_OK;
}
