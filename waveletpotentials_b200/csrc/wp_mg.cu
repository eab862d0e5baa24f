// wp_mg.cu -- solid-aware (cut-cell) fractional multigrid for -div(a grad p) = f with zero-flux
// walls, 3D and 2D, in FP32, FP64 and mixed precision (FP32 V-cycles inside FP64 iterative
// refinement).
//
// Reference behaviour: CuMultigridFrac3D (cuMultigridFrac3D.cu:9-134 hierarchy, :249-327 V-cycle),
// weighted Jacobi cuWjFrac3D_n (cuWeightedJacobi3D.cu:620-695), residual cuWjGetFracRes_3d_n
// (:1107-1181), relative residual GetFracRhs (:1384-1407), coarsest 50-sweep solve
// cuWjFrac3D_kernel_n (:1473-1545), cell restriction cuRestrict3D_p1_d{x,y,z} (cuRestrict3D.cu:801-970),
// face-fraction coarsening SolveP1Ax/Ay/Az (:972-1145), piecewise-constant prolongation
// cuProlongate3D_p1_* (cuProlongate3D.cu:353-424, 594-617), coarse spacing cuRestrictDx
// (cuMultigridFrac2D.cu:4-17); 2D: CuMultigridFrac2D (cuMultigridFrac2D.cu:28-215, coarsest = 10
// ordinary sweeps) and cuWeightedJacobi_frac_n (cuWeightedJacobi.cu:292-347).
//
// Operator: A v = sum_f cf (v - v_nb) over interior faces, cf = a_f * 2 / ((d_nb + d) d); a cell
// whose diagonal is <= 1e-12 is fixed to 0.  Kernels: one sweep / fused prolongation+sweep /
// fused residual+restriction per level (the reference uses 1 + 3 + 3 launches for the latter),
// a single-CTA coarsest solve, and FP64 defect / norm kernels for the refinement loop.
#include "wp_common.cuh"
#include "wp_tc.cuh"

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

namespace {

constexpr double kEps = 1e-12;
constexpr int kMaxLevels = 24;

template <typename T>
struct Lvl {
    int nx, ny, nz;
    const float* ax;
    const float* ay;
    const float* az;
    const float* fyc; // y-face fractions in cell layout: fyc[cell] = ay of the cell's lower y face
    const unsigned char* uni; // per (x, z) row, at [z nx + x]: 1 when every face fraction the row's
                              // stencils read (interior faces only) is exactly 1
    const T* glo[3];  // per-axis factor of the lower face, 0 at the wall
    const T* ghi[3];  // per-axis factor of the upper face, 0 at the wall
    const double* d[3];
    const float* rwz;  // restriction weight of fine plane z: (float)(d_z / (d_{2k} + d_{2k+1})), formed in FP64
};

// diag and off-diagonal sum of row (x,y,z) applied to v (optionally plus the prolonged coarse
// correction vc, i.e. v + P vc, piecewise constant)
template <typename T, typename TV, bool PROL>
__device__ __forceinline__ void row(const Lvl<T>& L, const TV* __restrict__ v, const TV* __restrict__ vc, int ncx,
                                    int ncy, int x, int y, int z, T& diag, T& off, T& vcen) {
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const long sxy = (long)nx * ny;
    const long i = y + (long)x * ny + z * sxy;
    auto V = [&](int xx, int yy, int zz, long ii) -> T {
        T r = (T)v[ii];
        if (PROL) r += (T)vc[(yy >> 1) + (long)(xx >> 1) * ncy + (long)(zz >> 1) * ncx * ncy];
        return r;
    };
    vcen = V(x, y, z, i);
    const long iax = y + (long)x * ny + (long)z * (nx + 1) * ny;
    const long iay = y + (long)x * (ny + 1) + (long)z * nx * (ny + 1);
    T dg = 0, od = 0, cf;
    if (y > 0) { cf = (T)L.ay[iay] * L.glo[1][y]; dg += cf; od -= cf * V(x, y - 1, z, i - 1); }
    if (y < ny - 1) { cf = (T)L.ay[iay + 1] * L.ghi[1][y]; dg += cf; od -= cf * V(x, y + 1, z, i + 1); }
    if (x > 0) { cf = (T)L.ax[iax] * L.glo[0][x]; dg += cf; od -= cf * V(x - 1, y, z, i - ny); }
    if (x < nx - 1) { cf = (T)L.ax[iax + ny] * L.ghi[0][x]; dg += cf; od -= cf * V(x + 1, y, z, i + ny); }
    if (z > 0) { cf = (T)L.az[i] * L.glo[2][z]; dg += cf; od -= cf * V(x, y, z - 1, i - sxy); }
    if (z < nz - 1) { cf = (T)L.az[i + sxy] * L.ghi[2][z]; dg += cf; od -= cf * V(x, y, z + 1, i + sxy); }
    diag = dg;
    off = od;
}

template <typename T, bool PROL>
__global__ void __launch_bounds__(256) jacobi_kernel(T* __restrict__ dst, const T* __restrict__ src, const T* __restrict__ f,
                                                     Lvl<T> L, T w, const T* __restrict__ vc, int ncx, int ncy) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (y >= L.ny || x >= L.nx) return;
    T dg, od, c;
    row<T, T, PROL>(L, src, vc, ncx, ncy, x, y, z, dg, od, c);
    const long i = y + (long)x * L.ny + (long)z * L.nx * L.ny;
    dst[i] = dg > (T)kEps ? ((T)1 - w) * c + w * (f[i] - od) / dg : (T)0;
}

// Column walker: the row of cell (x, y, z) for z = z0, z0+1, ... with the z neighbours and the
// z-face fraction carried in registers, so each v and az value of the column is loaded once;
// in-plane neighbours come through L1 (they are loaded by the neighbouring threads of the CTA).
template <typename T, typename TV, bool PROL>
struct ZCol {
    const Lvl<T>& L;
    const TV* __restrict__ v;
    const TV* __restrict__ vc;
    int ncx, ncy, x, y, z;
    long sxy, i, iax, iay, sax, say;
    T vm, vcur, az_lo, gxl, gxh, gyl, gyh;

    __device__ __forceinline__ T V(long ii, int xx, int yy, int zz) const {
        T r = (T)v[ii];
        if (PROL) r += (T)vc[(yy >> 1) + (long)(xx >> 1) * ncy + (long)(zz >> 1) * ncx * ncy];
        return r;
    }

    __device__ __forceinline__ ZCol(const Lvl<T>& L_, const TV* v_, const TV* vc_, int ncx_, int ncy_, int x_, int y_,
                                    int z0)
        : L(L_), v(v_), vc(vc_), ncx(ncx_), ncy(ncy_), x(x_), y(y_), z(z0) {
        sxy = (long)L.nx * L.ny;
        i = y + (long)x * L.ny + z0 * sxy;
        sax = (long)(L.nx + 1) * L.ny;
        say = (long)L.nx * (L.ny + 1);
        iax = y + (long)x * L.ny + z0 * sax;
        iay = y + (long)x * (L.ny + 1) + z0 * say;
        vm = z0 > 0 ? V(i - sxy, x, y, z0 - 1) : (T)0;
        vcur = V(i, x, y, z0);
        az_lo = z0 > 0 ? (T)L.az[i] : (T)0;
        gxl = L.glo[0][x];
        gxh = L.ghi[0][x];
        gyl = L.glo[1][y];
        gyh = L.ghi[1][y];
    }

    // diag, off-diagonal sum and centre value of the current cell; then advances one plane
    __device__ __forceinline__ void step(T& dg, T& od, T& c) {
        const int nx = L.nx, ny = L.ny, nz = L.nz;
        T d = 0, o = 0, cf;
        if (y > 0) { cf = (T)L.ay[iay] * gyl; d += cf; o -= cf * V(i - 1, x, y - 1, z); }
        if (y < ny - 1) { cf = (T)L.ay[iay + 1] * gyh; d += cf; o -= cf * V(i + 1, x, y + 1, z); }
        if (x > 0) { cf = (T)L.ax[iax] * gxl; d += cf; o -= cf * V(i - ny, x - 1, y, z); }
        if (x < nx - 1) { cf = (T)L.ax[iax + ny] * gxh; d += cf; o -= cf * V(i + ny, x + 1, y, z); }
        T vp = 0, az_hi = 0;
        if (z > 0) { cf = az_lo * L.glo[2][z]; d += cf; o -= cf * vm; }
        if (z < nz - 1) {
            vp = V(i + sxy, x, y, z + 1);
            az_hi = (T)L.az[i + sxy];
            cf = az_hi * L.ghi[2][z];
            d += cf;
            o -= cf * vp;
        }
        dg = d;
        od = o;
        c = vcur;
        vm = vcur;
        vcur = vp;
        az_lo = az_hi;
        i += sxy;
        iax += sax;
        iay += say;
        ++z;
    }
};

template <typename T, bool PROL>
__global__ void __launch_bounds__(256) jacobi_z_kernel(T* __restrict__ dst, const T* __restrict__ src,
                                                       const T* __restrict__ f, Lvl<T> L, T w,
                                                       const T* __restrict__ vc, int ncx, int ncy, int zc) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y;
    const int z0 = blockIdx.z * zc, z1 = min(z0 + zc, L.nz);
    if (y >= L.ny || x >= L.nx || z0 >= z1) return;
    ZCol<T, T, PROL> col(L, src, vc, ncx, ncy, x, y, z0);
    for (int z = z0; z < z1; ++z) {
        const long i = col.i;
        T dg, od, c;
        col.step(dg, od, c);
        dst[i] = dg > (T)kEps ? ((T)1 - w) * c + w * (f[i] - od) / dg : (T)0;
    }
}

// ------------------------------------------------------------------ quad kernels
// The same operator with each thread owning four consecutive cells along y (y0 = 4k; needs
// ny % 4 == 0): v, f, ax, az and the cell-laid y fractions move as 128-bit loads (two 64-bit-pair
// loads for FP64), the z neighbours and z-face fractions of the column stay in registers, and the
// x neighbours come through L1 from the adjacent rows.  Per cell the arithmetic (terms and their
// order) is that of `row` / ZCol.
template <typename T>
struct Q4 {
    T a[4];
};

__device__ __forceinline__ Q4<float> ld4(const float* p) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    return {{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ Q4<double> ld4(const double* p) {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *reinterpret_cast<const double2*>(p + 2);
    return {{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float* p, const Q4<float>& v) {
    *reinterpret_cast<float4*>(p) = make_float4(v.a[0], v.a[1], v.a[2], v.a[3]);
}
__device__ __forceinline__ void st4(double* p, const Q4<double>& v) {
    *reinterpret_cast<double2*>(p) = make_double2(v.a[0], v.a[1]);
    *reinterpret_cast<double2*>(p + 2) = make_double2(v.a[2], v.a[3]);
}
template <typename T, typename S>
__device__ __forceinline__ Q4<T> cvt4(const Q4<S>& v) {
    return {{(T)v.a[0], (T)v.a[1], (T)v.a[2], (T)v.a[3]}};
}
template <typename T>
__device__ __forceinline__ Q4<T> zero4() {
    return {{(T)0, (T)0, (T)0, (T)0}};
}

// Loads of data that another CTA of the same grid may have written earlier in the grid's life (the
// persistent coarse-level kernel): cache-global (L2) loads, never a possibly stale L1 line or the
// non-coherent read-only path.  CG = false: ordinary loads.
template <bool CG>
__device__ __forceinline__ Q4<float> ldq(const float* p) {
    if constexpr (CG) {
        const float4 t = __ldcg(reinterpret_cast<const float4*>(p));
        return {{t.x, t.y, t.z, t.w}};
    } else {
        return ld4(p);
    }
}
template <bool CG>
__device__ __forceinline__ Q4<double> ldq(const double* p) {
    if constexpr (CG) {
        const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldcg(reinterpret_cast<const double2*>(p + 2));
        return {{a.x, a.y, b.x, b.y}};
    } else {
        return ld4(p);
    }
}
template <bool CG, typename V>
__device__ __forceinline__ V ld1(const V* p) {
    if constexpr (CG) return __ldcg(p);
    else return *p;
}

// Walker over the quad (x, y0..y0+3) of a column, z = z0, z0+1, ...  CG: v through L2 (see ldq).
template <typename T, typename TV, bool CG = false>
struct QCol {
    const Lvl<T>& L;
    const TV* __restrict__ v;
    int x, y0, z;
    long sxy, sax, i, iax;
    bool xm, xp, ym, yp;
    unsigned char un; // row flag of plane z
    T gxl, gxh, gyl[4], gyh[4];
    Q4<T> vm, vc, azl;

    __device__ __forceinline__ QCol(const Lvl<T>& L_, const TV* v_, int x_, int y0_, int z0)
        : L(L_), v(v_), x(x_), y0(y0_), z(z0) {
        sxy = (long)L.nx * L.ny;
        sax = (long)(L.nx + 1) * L.ny;
        i = y0 + (long)x * L.ny + z0 * sxy;
        iax = y0 + (long)x * L.ny + z0 * sax;
        xm = x > 0;
        xp = x < L.nx - 1;
        ym = y0 > 0;
        yp = y0 + 4 < L.ny;
        gxl = L.glo[0][x];
        gxh = L.ghi[0][x];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            gyl[k] = L.glo[1][y0 + k];
            gyh[k] = L.ghi[1][y0 + k];
        }
        vm = z0 > 0 ? cvt4<T>(ldq<CG>(v + i - sxy)) : zero4<T>();
        vc = cvt4<T>(ldq<CG>(v + i));
        azl = z0 > 0 ? cvt4<T>(ld4(L.az + i)) : zero4<T>();
        un = z0 < L.nz ? L.uni[(long)z0 * L.nx + x] : 0;
    }

    __device__ __forceinline__ void step(Q4<T>& dg, Q4<T>& od, Q4<T>& c) {
        Q4<T> vp = zero4<T>();
        if (z < L.nz - 1) vp = cvt4<T>(ldq<CG>(v + i + sxy));
        step_with(dg, od, c, vp);
    }

    // one step with the next plane's centre quad vp supplied by the caller (zero above the top)
    __device__ __forceinline__ void step_with(Q4<T>& dg, Q4<T>& od, Q4<T>& c, const Q4<T> vp) {
        const int ny = L.ny, nz = L.nz;
        const bool zp = z < nz - 1;
        // a row whose faces are all exactly 1 reads no fractions (the same values, without the traffic)
        const bool u = un != 0;
        un = zp ? L.uni[(long)(z + 1) * L.nx + x] : 0;
        const T vym = ym ? (T)ld1<CG>(v + i - 1) : (T)0;
        const T vyp = yp ? (T)ld1<CG>(v + i + 4) : (T)0;
        const Q4<T> vxm = xm ? cvt4<T>(ldq<CG>(v + i - ny)) : zero4<T>();
        const Q4<T> vxp = xp ? cvt4<T>(ldq<CG>(v + i + ny)) : zero4<T>();
        Q4<T> azu = zero4<T>();
        const T gzl = L.glo[2][z], gzh = L.ghi[2][z];
        if (u && xm && xp && z > 0 && zp) {
            // uniform interior row: each face coefficient is its spacing factor (1 x factor), every
            // neighbour exists except y ones at the ends of the row
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                T d = 0, o = 0;
                if (k > 0 || ym) { d += gyl[k]; o -= gyl[k] * (k > 0 ? vc.a[k - 1] : vym); }
                if (k < 3 || yp) { d += gyh[k]; o -= gyh[k] * (k < 3 ? vc.a[k + 1] : vyp); }
                d += gxl; o -= gxl * vxm.a[k];
                d += gxh; o -= gxh * vxp.a[k];
                d += gzl; o -= gzl * vm.a[k];
                d += gzh; o -= gzh * vp.a[k];
                dg.a[k] = d;
                od.a[k] = o;
                c.a[k] = vc.a[k];
            }
            azu = Q4<T>{{(T)1, (T)1, (T)1, (T)1}};
        } else {
            Q4<float> fyl, fxl, fxu = zero4<float>();
            float fyu = 0.f;
            if (u) {
                fyl = fxl = Q4<float>{{1.f, 1.f, 1.f, 1.f}};
                if (yp) fyu = 1.f;
                if (xp) fxu = fxl;
                if (zp) azu = Q4<T>{{(T)1, (T)1, (T)1, (T)1}};
            } else {
                fyl = ld4(L.fyc + i);
                if (yp) fyu = L.fyc[i + 4];
                fxl = ld4(L.ax + iax);
                if (xp) fxu = ld4(L.ax + iax + ny);
                if (zp) azu = cvt4<T>(ld4(L.az + i + sxy));
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int y = y0 + k;
                T d = 0, o = 0, cf;
                if (y > 0) { cf = (T)fyl.a[k] * gyl[k]; d += cf; o -= cf * (k > 0 ? vc.a[k - 1] : vym); }
                if (y < ny - 1) { cf = (T)(k < 3 ? fyl.a[k + 1] : fyu) * gyh[k]; d += cf; o -= cf * (k < 3 ? vc.a[k + 1] : vyp); }
                if (xm) { cf = (T)fxl.a[k] * gxl; d += cf; o -= cf * vxm.a[k]; }
                if (xp) { cf = (T)fxu.a[k] * gxh; d += cf; o -= cf * vxp.a[k]; }
                if (z > 0) { cf = azl.a[k] * gzl; d += cf; o -= cf * vm.a[k]; }
                if (zp) { cf = azu.a[k] * gzh; d += cf; o -= cf * vp.a[k]; }
                dg.a[k] = d;
                od.a[k] = o;
                c.a[k] = vc.a[k];
            }
        }
        vm = vc;
        vc = vp;
        azl = azu;
        i += sxy;
        iax += sax;
        ++z;
    }
};

// y-quad index of a thread: q = x * (ny / 4) + yq over one z-plane.  ACC: the swept values are not
// stored but added to the FP64 iterate p64 (the refinement update fused into the last sweep of a
// correction cycle, add_correction_kernel's arithmetic).
template <typename T, bool ACC = false, bool CG = false>
__device__ __forceinline__ void jacobi_q_body(T* __restrict__ dst, const T* __restrict__ src, const T* __restrict__ f,
                                              const Lvl<T>& L, T w, int zc, double* __restrict__ p64, int bx, int by,
                                              int tid) {
    const int nq = L.ny >> 2;
    const long q = (long)bx * 256 + tid;
    const int z0 = by * zc, z1 = min(z0 + zc, L.nz);
    if (q >= (long)L.nx * nq || z0 >= z1) return;
    const int x = (int)(q / nq), y0 = (int)(q - (long)x * nq) * 4;
    QCol<T, T, CG> col(L, src, x, y0, z0);
    for (int z = z0; z < z1; ++z) {
        const long i = col.i;
        Q4<T> dg, od, c;
        col.step(dg, od, c);
        const Q4<T> fv = ldq<CG>(f + i);
        Q4<T> out;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            out.a[k] = dg.a[k] > (T)kEps ? ((T)1 - w) * c.a[k] + w * (fv.a[k] - od.a[k]) / dg.a[k] : (T)0;
        if (ACC) {
            Q4<double> pv = ldq<CG>(p64 + i);
#pragma unroll
            for (int k = 0; k < 4; ++k) pv.a[k] += (double)out.a[k];
            st4(p64 + i, pv);
        } else {
            st4(dst + i, out);
        }
    }
}

// The first sweep from v = 0: every neighbour and the centre are 0, so the sweep is
// (1 - w) 0 + w (f - 0) / diag, which reads only f and (outside uniform rows) the fractions for the
// diagonal -- the same value as jacobi_q_body on a zeroed v, with no v to clear or read.
template <typename T, bool CG = false>
__device__ __forceinline__ void jacobi0_q_body(T* __restrict__ dst, const T* __restrict__ f, const Lvl<T>& L, T w,
                                               int zc, int bx, int by, int tid) {
    const int nq = L.ny >> 2;
    const long q = (long)bx * 256 + tid;
    const int z0 = by * zc, z1 = min(z0 + zc, L.nz);
    if (q >= (long)L.nx * nq || z0 >= z1) return;
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const int x = (int)(q / nq), y0 = (int)(q - (long)x * nq) * 4;
    const long sxy = (long)nx * ny, sax = (long)(nx + 1) * ny;
    long i = y0 + (long)x * ny + z0 * sxy, iax = y0 + (long)x * ny + z0 * sax;
    const bool xm = x > 0, xp = x < nx - 1, yp = y0 + 4 < ny;
    const T gxl = L.glo[0][x], gxh = L.ghi[0][x];
    T gyl[4], gyh[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        gyl[k] = L.glo[1][y0 + k];
        gyh[k] = L.ghi[1][y0 + k];
    }
    unsigned char un = L.uni[(long)z0 * nx + x];
    Q4<T> azl = z0 > 0 ? cvt4<T>(ld4(L.az + i)) : zero4<T>();
    for (int z = z0; z < z1; ++z) {
        const bool zp = z < nz - 1;
        const bool u = un != 0;
        un = zp ? L.uni[(long)(z + 1) * nx + x] : 0;
        Q4<float> fyl, fxl, fxu = zero4<float>();
        float fyu = 0.f;
        Q4<T> azu = zero4<T>();
        if (u) {
            fyl = fxl = Q4<float>{{1.f, 1.f, 1.f, 1.f}};
            if (yp) fyu = 1.f;
            if (xp) fxu = fxl;
            if (zp) azu = Q4<T>{{(T)1, (T)1, (T)1, (T)1}};
        } else {
            fyl = ld4(L.fyc + i);
            if (yp) fyu = L.fyc[i + 4];
            fxl = ld4(L.ax + iax);
            if (xp) fxu = ld4(L.ax + iax + ny);
            if (zp) azu = cvt4<T>(ld4(L.az + i + sxy));
        }
        const T gzl = L.glo[2][z], gzh = L.ghi[2][z];
        const Q4<T> fv = ldq<CG>(f + i);
        Q4<T> out;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int y = y0 + k;
            T d = 0;
            if (y > 0) d += (T)fyl.a[k] * gyl[k];
            if (y < ny - 1) d += (T)(k < 3 ? fyl.a[k + 1] : fyu) * gyh[k];
            if (xm) d += (T)fxl.a[k] * gxl;
            if (xp) d += (T)fxu.a[k] * gxh;
            if (z > 0) d += azl.a[k] * gzl;
            if (zp) d += azu.a[k] * gzh;
            out.a[k] = d > (T)kEps ? ((T)1 - w) * (T)0 + w * (fv.a[k] - (T)0) / d : (T)0;
        }
        st4(dst + i, out);
        azl = azu;
        i += sxy;
        iax += sax;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) jacobi0_q_kernel(T* __restrict__ dst, const T* __restrict__ f, Lvl<T> L, T w,
                                                        int zc) {
    wp_pdl_enter();
    jacobi0_q_body<T>(dst, f, L, w, zc, blockIdx.x, blockIdx.y, threadIdx.x);
}

// register-allocation variants of the same sweep (the autotuner picks one per level): default
// limits, and at least 3 or 4 resident 256-thread CTAs per SM
template <typename T, bool ACC = false>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 2 : 1) jacobi_q_kernel(T* __restrict__ dst, const T* __restrict__ src,
                                                       const T* __restrict__ f, Lvl<T> L, T w, int zc,
                                                       double* __restrict__ p64 = nullptr) {
    wp_pdl_enter();
    jacobi_q_body<T, ACC>(dst, src, f, L, w, zc, p64, blockIdx.x, blockIdx.y, threadIdx.x);
}
template <typename T, int MINB, bool ACC = false>
__global__ void __launch_bounds__(256, MINB) jacobi_q_mb_kernel(T* __restrict__ dst, const T* __restrict__ src,
                                                                const T* __restrict__ f, Lvl<T> L, T w, int zc,
                                                                double* __restrict__ p64 = nullptr) {
    wp_pdl_enter();
    jacobi_q_body<T, ACC>(dst, src, f, L, w, zc, p64, blockIdx.x, blockIdx.y, threadIdx.x);
}

// The one-sweep quad kernel with its streaming loads issued ahead: every thread keeps a private
// ring of JP_DEPTH planes in shared memory and fills it with cp.async (16-byte, L2-only) copies of the
// next planes' centre quad v(z+1) and right-hand side f(z), JP_DEPTH - 1 planes before it uses them,
// so each warp has several planes of DRAM reads in flight without holding them in registers.  The
// arithmetic per cell is QCol's (step_with).  No thread reads another's ring slots: no barriers.
constexpr int JP_DEPTH = 4;
constexpr size_t jp_smem_bytes(bool acc) { return (size_t)JP_DEPTH * 256 * 16 * (acc ? 4 : 2); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(wptc::smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ACC: the swept values are added to the FP64 iterate p64 (jacobi_q_body's ACC form), whose quads
// stream through the ring as well.
template <bool ACC = false>
__global__ void __launch_bounds__(256, 3) jacobi_qp_kernel(float* __restrict__ dst, const float* __restrict__ src,
                                                           const float* __restrict__ f, Lvl<float> L, float w,
                                                           int zc, double* __restrict__ p64) {
    wp_pdl_enter();
    // dynamic shared memory: ring_v | ring_f (JP_DEPTH x 256 float4 each) | ring_p (ACC: JP_DEPTH x 512 double2)
    extern __shared__ __align__(16) float4 jp_smem[];
    float4 (*ring_v)[256] = reinterpret_cast<float4 (*)[256]>(jp_smem);
    float4 (*ring_f)[256] = reinterpret_cast<float4 (*)[256]>(jp_smem + JP_DEPTH * 256);
    double2 (*ring_p)[512] = reinterpret_cast<double2 (*)[512]>(jp_smem + 2 * JP_DEPTH * 256);
    const int tid = threadIdx.x;
    const int nq = L.ny >> 2;
    const long q = (long)blockIdx.x * 256 + tid;
    const int z0 = blockIdx.y * zc, z1 = min(z0 + zc, L.nz);
    if (q >= (long)L.nx * nq || z0 >= z1) return;
    const int x = (int)(q / nq), y0 = (int)(q - (long)x * nq) * 4;
    const long sxy = (long)L.nx * L.ny;
    const long ibase = y0 + (long)x * L.ny;
    auto issue = [&](int p) {
        const int slot = (p - z0) % JP_DEPTH;
        if (p < z1) {
            if (p + 1 < L.nz) cp_async16(&ring_v[slot][tid], src + ibase + (long)(p + 1) * sxy);
            cp_async16(&ring_f[slot][tid], f + ibase + (long)p * sxy);
            if constexpr (ACC) {
                cp_async16(&ring_p[slot][2 * tid], p64 + ibase + (long)p * sxy);
                cp_async16(&ring_p[slot][2 * tid + 1], p64 + ibase + (long)p * sxy + 2);
            }
        }
        cp_async_commit();  // one group per plane (empty past the chunk) keeps the count uniform
    };
    for (int p = z0; p < z0 + JP_DEPTH - 1; ++p) issue(p);
    QCol<float, float> col(L, src, x, y0, z0);
    for (int z = z0; z < z1; ++z) {
        issue(z + JP_DEPTH - 1);
        cp_async_wait<JP_DEPTH - 1>();  // the group of plane z has landed
        const int slot = (z - z0) % JP_DEPTH;
        const long i = col.i;
        Q4<float> vp = zero4<float>();
        if (z < L.nz - 1) {
            const float4 t = ring_v[slot][tid];
            vp = Q4<float>{{t.x, t.y, t.z, t.w}};
        }
        const float4 tf = ring_f[slot][tid];
        const Q4<float> fv{{tf.x, tf.y, tf.z, tf.w}};
        Q4<float> dg, od, c;
        col.step_with(dg, od, c, vp);
        Q4<float> out;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            out.a[k] = dg.a[k] > (float)kEps ? (1.f - w) * c.a[k] + w * (fv.a[k] - od.a[k]) / dg.a[k] : 0.f;
        if constexpr (ACC) {
            const double2 a = ring_p[slot][2 * tid], b = ring_p[slot][2 * tid + 1];
            const Q4<double> pv{{a.x + (double)out.a[0], a.y + (double)out.a[1], b.x + (double)out.a[2],
                                 b.y + (double)out.a[3]}};
            st4(p64 + i, pv);
        } else {
            st4(dst + i, out);
        }
    }
    cp_async_wait<0>();
}

// Two weighted-Jacobi sweeps in one pass (temporal blocking along z).  A CTA owns an interior tile
// of J2_R rows x J2_Q quads and a z-chunk; its 288 threads cover the tile plus a one-row /
// one-quad halo.  Walking up the chunk, every thread computes the first sweep of its quad at plane z
// (QCol, as jacobi_q_kernel) into a three-plane shared ring; after a barrier the interior threads
// compute the second sweep at plane z - 1 from the ring (the same terms in the same order, with the
// face fractions re-read through L1).  The first sweep runs one plane beyond each end of the chunk,
// so every second-sweep stencil finds its z neighbours.  Two sweeps then cost one read of v, f and
// the fractions instead of two.
constexpr int J2_R = 14, J2_Q = 16;
constexpr int J2_RH = J2_R + 2, J2_QH = J2_Q + 2;
constexpr int J2_THREADS = J2_RH * J2_QH;
constexpr int J2_PITCH = J2_QH * 4 + 4;  // row pitch of the ring (elements); the pad staggers banks

template <typename T>
__device__ __forceinline__ void jacobi2_body(T* __restrict__ dst, const T* __restrict__ src, const T* __restrict__ f,
                                             const Lvl<T>& L, T w, int zc, int nty, T (*s1)[J2_RH][J2_PITCH]) {
    const int nq = L.ny >> 2;
    const int tile_x = blockIdx.x / nty, tile_y = blockIdx.x - tile_x * nty;
    const int hr = threadIdx.x / J2_QH, hq = threadIdx.x - hr * J2_QH;
    const int x = tile_x * J2_R - 1 + hr, yq = tile_y * J2_Q - 1 + hq;
    const bool indom = x >= 0 && x < L.nx && yq >= 0 && yq < nq;
    const bool interior = indom && hr >= 1 && hr <= J2_R && hq >= 1 && hq <= J2_Q;
    const int z0 = blockIdx.y * zc, z1 = min(z0 + zc, L.nz);
    const int zs = max(z0 - 1, 0), ze = min(z1, L.nz - 1);
    const int xc = indom ? x : 0, y0 = indom ? 4 * yq : 0;
    QCol<T, T> col(L, src, xc, y0, zs);
    const long sxy = (long)L.nx * L.ny, sax = (long)(L.nx + 1) * L.ny;
    const int ny = L.ny, nz = L.nz;
    for (int z = zs; z <= z1; ++z) {
        if (z <= ze) {
            Q4<T> v1 = zero4<T>();
            if (indom) {
                const long i = col.i;
                Q4<T> dg, od, c;
                col.step(dg, od, c);
                const Q4<T> fv = ld4(f + i);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    v1.a[k] = dg.a[k] > (T)kEps ? ((T)1 - w) * c.a[k] + w * (fv.a[k] - od.a[k]) / dg.a[k] : (T)0;
            }
            T* row = &s1[z % 3][hr][hq * 4];
#pragma unroll
            for (int k = 0; k < 4; ++k) row[k] = v1.a[k];
        }
        __syncthreads();
        const int zz = z - 1;
        if (interior && zz >= z0 && zz < z1) {
            const T* cm = &s1[zz % 3][hr][hq * 4];
            const T* cxm = &s1[zz % 3][hr - 1][hq * 4];
            const T* cxp = &s1[zz % 3][hr + 1][hq * 4];
            const T* czm = &s1[(zz + 2) % 3][hr][hq * 4];  // plane zz - 1
            const T* czp = &s1[(zz + 1) % 3][hr][hq * 4];  // plane zz + 1
            const long i = y0 + (long)x * ny + zz * sxy;
            const long iax = y0 + (long)x * ny + zz * sax;
            const Q4<float> fyl = ld4(L.fyc + i);
            const bool yp = y0 + 4 < ny;
            const float fyu = yp ? L.fyc[i + 4] : 0.f;
            const Q4<float> fxl = ld4(L.ax + iax);
            const Q4<float> fxu = col.xp ? ld4(L.ax + iax + ny) : zero4<float>();
            const Q4<T> azl = zz > 0 ? cvt4<T>(ld4(L.az + i)) : zero4<T>();
            const bool zp = zz < nz - 1;
            const Q4<T> azu = zp ? cvt4<T>(ld4(L.az + i + sxy)) : zero4<T>();
            const Q4<T> fv = ld4(f + i);
            const T gzl = L.glo[2][zz], gzh = L.ghi[2][zz];
            const T vym = cm[-1], vyp = cm[4];
            Q4<T> out;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int y = y0 + k;
                T d = 0, o = 0, cf;
                if (y > 0) { cf = (T)fyl.a[k] * col.gyl[k]; d += cf; o -= cf * (k > 0 ? cm[k - 1] : vym); }
                if (y < ny - 1) { cf = (T)(k < 3 ? fyl.a[k + 1] : fyu) * col.gyh[k]; d += cf; o -= cf * (k < 3 ? cm[k + 1] : vyp); }
                if (col.xm) { cf = (T)fxl.a[k] * col.gxl; d += cf; o -= cf * cxm[k]; }
                if (col.xp) { cf = (T)fxu.a[k] * col.gxh; d += cf; o -= cf * cxp[k]; }
                if (zz > 0) { cf = azl.a[k] * gzl; d += cf; o -= cf * czm[k]; }
                if (zp) { cf = azu.a[k] * gzh; d += cf; o -= cf * czp[k]; }
                out.a[k] = d > (T)kEps ? ((T)1 - w) * cm[k] + w * (fv.a[k] - o) / d : (T)0;
            }
            st4(dst + i, out);
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(J2_THREADS, sizeof(T) == 4 ? 2 : 1)
    jacobi2_q_kernel(T* __restrict__ dst, const T* __restrict__ src, const T* __restrict__ f, Lvl<T> L, T w, int zc,
                     int nty) {
    __shared__ __align__(16) T s1[3][J2_RH][J2_PITCH];
    jacobi2_body<T>(dst, src, f, L, w, zc, nty, s1);
}

// TMA-staged Jacobi sweep.  Persistent CTAs (one per SM) split the (x-tile, z) planes of the level
// evenly; a tile is R whole x rows (all y).  Per plane a single thread issues contiguous row copies
// on the TMA engine (cp.async.bulk) into a 4-slot ring: the v rows of the tile and its two x
// neighbours, and the f, y-face (cell-laid), x-face (R + 1 rows) and z-face rows.  Plane z is
// computed from the slots of z-1, z and z+1 while z+2 is in flight; after a block barrier the slot of
// z-1 receives plane z+3.  Compute reads only shared memory (128-bit, conflict-free) and writes the
// result with 128-bit stores, so the DRAM stream is the copies alone.  Per cell the arithmetic is
// QCol::step's (same terms, same order).
constexpr int TS_STAGES = 4;
constexpr int TS_THREADS = 256;

__host__ __device__ inline int ts_stage_floats(int R, int ny) { return (5 * R + 3) * ny; }

// rows per tile so that four slots fit in 100 KB of shared memory (two CTAs per SM)
inline int ts_rows(int nx, int ny) {
    int r = ((100 * 1024) / (4 * TS_STAGES * ny) - 3) / 5;
    return std::max(1, std::min(r, nx));
}
inline size_t ts_smem_bytes(int R, int ny) { return ((size_t)ts_stage_floats(R, ny) * TS_STAGES + 2 * ny) * 4; }

__global__ void __launch_bounds__(TS_THREADS, 2)
    jacobi_ts_kernel(float* __restrict__ dst, const float* __restrict__ src, const float* __restrict__ f,
                     Lvl<float> L, float w, int R, int* err) {
    using namespace wptc;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long bars[TS_STAGES];
    float* sm = reinterpret_cast<float*>(smem_raw);
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const int stg = ts_stage_floats(R, ny);
    const long sxy = (long)nx * ny, sax = (long)(nx + 1) * ny;
    const int ntiles = (nx + R - 1) / R;
    const long W = (long)ntiles * nz;
    const long u0 = W * blockIdx.x / gridDim.x, u1 = W * (blockIdx.x + 1) / gridDim.x;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // y-face geometry of the level, read once per CTA
    float* gyl = sm + (size_t)TS_STAGES * stg;
    float* gyh = gyl + ny;
    for (int y = tid; y < ny; y += TS_THREADS) {
        gyl[y] = L.glo[1][y];
        gyh[y] = L.ghi[1][y];
    }
    if (tid == 0) {
        for (int s = 0; s < TS_STAGES; ++s) mbar_init(smem_u32(&bars[s]), 1);
        mbar_init_fence();
    }
    __syncthreads();
    uint32_t uses[TS_STAGES] = {0, 0, 0, 0};
    const int nqr = ny >> 2;
    // slot regions: v (R + 2 rows, row 0 = x0 - 1) | f (R) | ax (R + 1) | fyc (R) | az (R)
    auto sv = [&](int p) { return sm + (size_t)(p % TS_STAGES) * stg; };
    auto sf = [&](int p) { return sv(p) + (R + 2) * ny; };
    auto sa = [&](int p) { return sf(p) + R * ny; };
    auto sy = [&](int p) { return sa(p) + (R + 1) * ny; };
    auto sz = [&](int p) { return sy(p) + R * ny; };
    bool ok = true;
    long u = u0;
    while (u < u1 && ok) {
        const int tile = (int)(u / nz);
        const int zb = (int)(u - (long)tile * nz);
        const int ze = (int)min((long)nz, zb + (u1 - u));
        const int x0 = tile * R, rows = min(R, nx - x0);
        const int plast = min(ze, nz - 1);
        // warp 0 issues the plane's row copies, one per lane, after lane 0 posted the byte count
        auto issue = [&](int p) {
            const int s = p % TS_STAGES;
            if (warp == 0) {
                const uint32_t bar = smem_u32(&bars[s]);
                const int xv0 = max(x0 - 1, 0), xv1 = min(x0 + rows + 1, nx), xa1 = min(x0 + rows + 1, nx + 1);
                const int nv = xv1 - xv0, ncp = nv + 3 * rows + (xa1 - x0);
                const uint32_t rb = (uint32_t)ny * 4u;
                if (lane == 0) mbar_expect_tx(bar, rb * (uint32_t)ncp);
                __syncwarp();
                for (int j = lane; j < ncp; j += 32) {
                    const float* g;
                    float* d;
                    if (j < nv) {
                        const int x = xv0 + j;
                        g = src + (long)x * ny + p * sxy;
                        d = sv(p) + (x - x0 + 1) * ny;
                    } else if (j < nv + 3 * rows) {
                        const int k = (j - nv) / rows, r = (j - nv) - k * rows;
                        const long o = (long)(x0 + r) * ny + p * sxy;
                        g = k == 0 ? f + o : k == 1 ? L.fyc + o : L.az + o;
                        d = (k == 0 ? sf(p) : k == 1 ? sy(p) : sz(p)) + r * ny;
                    } else {
                        const int x = x0 + (j - nv - 3 * rows);
                        g = L.ax + (long)x * ny + p * sax;
                        d = sa(p) + (x - x0) * ny;
                    }
                    bulk_load(smem_u32(d), g, rb, bar);
                }
            }
            uses[s] += 1;
        };
        auto wait = [&](int p) {
            return mbar_wait(smem_u32(&bars[p % TS_STAGES]), (uses[p % TS_STAGES] - 1) & 1, err);
        };
        for (int p = max(zb - 1, 0); p <= min(plast, zb + 2); ++p) issue(p);
        if (zb > 0) ok = wait(zb - 1) && ok;
        ok = wait(zb) && ok;
        for (int z = zb; z < ze; ++z) {
            const bool zp = z < nz - 1;
            if (zp) ok = wait(z + 1) && ok;
            if (!__syncthreads_and(ok)) {
                ok = false;
                break;
            }
            const float* vm = sv(z > 0 ? z - 1 : z);
            const float* vc = sv(z);
            const float* vp = sv(zp ? z + 1 : z);
            const float* fz = sf(z);
            const float* ax = sa(z);
            const float* fy = sy(z);
            const float* azl = sz(z);
            const float* azu = sz(zp ? z + 1 : z);
            const float gzl = L.glo[2][z], gzh = L.ghi[2][z];
            for (int q = tid; q < rows * nqr; q += TS_THREADS) {
                const int r = q / nqr, y0 = (q - r * nqr) * 4;
                const int x = x0 + r;
                const int o = r * ny + y0;         // row r of the f / fyc / az / lower-ax regions
                const int oc = (r + 1) * ny + y0;  // the cell's row in the v region
                const Q4<float> c = ld4(vc + oc);
                const Q4<float> vxm = ld4(vc + oc - ny), vxp = ld4(vc + oc + ny);
                const Q4<float> vzm = ld4(vm + oc), vzp = ld4(vp + oc);
                const Q4<float> fv = ld4(fz + o);
                const Q4<float> fyl = ld4(fy + o), fxl = ld4(ax + o), fxu = ld4(ax + o + ny);
                const Q4<float> al = ld4(azl + o), au = ld4(azu + o);
                const bool ym = y0 > 0, yp = y0 + 4 < ny, xm = x > 0, xp = x < nx - 1;
                const float vym = ym ? vc[oc - 1] : 0.f, vyp = yp ? vc[oc + 4] : 0.f;
                const float fyu = yp ? fy[o + 4] : 0.f;
                const float gxl = L.glo[0][x], gxh = L.ghi[0][x];
                Q4<float> out;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int y = y0 + k;
                    float d = 0.f, od = 0.f, cf;
                    if (y > 0) { cf = fyl.a[k] * gyl[y]; d += cf; od -= cf * (k > 0 ? c.a[k - 1] : vym); }
                    if (y < ny - 1) { cf = (k < 3 ? fyl.a[k + 1] : fyu) * gyh[y]; d += cf; od -= cf * (k < 3 ? c.a[k + 1] : vyp); }
                    if (xm) { cf = fxl.a[k] * gxl; d += cf; od -= cf * vxm.a[k]; }
                    if (xp) { cf = fxu.a[k] * gxh; d += cf; od -= cf * vxp.a[k]; }
                    if (z > 0) { cf = al.a[k] * gzl; d += cf; od -= cf * vzm.a[k]; }
                    if (zp) { cf = au.a[k] * gzh; d += cf; od -= cf * vzp.a[k]; }
                    out.a[k] = d > (float)kEps ? (1.f - w) * c.a[k] + w * (fv.a[k] - od) / d : 0.f;
                }
                st4(dst + y0 + (long)x * ny + z * sxy, out);
            }
            __syncthreads();
            if (z + 3 <= plast) issue(z + 3);
        }
        u += ze - zb;
    }
    if (!ok && tid == 0) {
        // a wait gave up: let the copies still in flight land before the CTA's shared memory goes
        for (int s = 0; s < TS_STAGES; ++s)
            if (uses[s]) mbar_wait(smem_u32(&bars[s]), (uses[s] - 1) & 1, err);
    }
}

// Fused residual + restriction on quads: lanes 2k and 2k+1 own the fine rows x0 = 2 cx and x0 + 1 of
// the quad y0..y0+3 (coarse cells cy = y0/2, y0/2 + 1); each walks both fine z children of every
// coarse plane and sums its y pairs in registers, and a lane shuffle adds the two rows:
// ((x0,y) + (x0,y+1)) + ((x0+1,y) + (x0+1,y+1)), each child carrying (0 + w_z0 r_z0) + w_z1 r_z1,
// the order of resid_restrict_z_kernel.
template <typename T, bool CG = false>
__device__ __forceinline__ void resid_restrict_q_body(T* __restrict__ fc, const T* __restrict__ v,
                                                      const T* __restrict__ f, const Lvl<T>& L, int ncx, int ncy,
                                                      int ncz, int czc, int bx, int by, int tid) {
    const int nq = L.ny >> 2;
    const long q = (long)bx * 256 + tid;
    const int cz0 = by * czc, cz1 = min(cz0 + czc, ncz);
    const long pair = q >> 1;
    const int xpar = (int)(q & 1);
    // whole warps stay together for the shuffle; lanes past the grid end only idle along
    const bool live_pair = pair < (long)ncx * nq && cz0 < cz1;
    const int cx = live_pair ? (int)(pair / nq) : 0;
    const int y0 = live_pair ? (int)(pair - (long)cx * nq) * 4 : 0;
    const int x0 = 2 * cx;
    const bool two = x0 + 1 < L.nx;
    const bool mine = live_pair && (xpar == 0 || two);
    const int x = mine ? x0 + xpar : x0;
    T wxy[4];
    {
        const double sx = L.d[0][x0] + (two ? L.d[0][x0 + 1] : 0.0);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int y = y0 + k, yb = y & ~1;
            const double sy = L.d[1][yb] + (yb + 1 < L.ny ? L.d[1][yb + 1] : 0.0);
            wxy[k] = mine ? (T)(L.d[1][y] / sy * (L.d[0][x] / sx)) : (T)0;
        }
    }
    QCol<T, T, CG> col(L, v, x, y0, live_pair ? 2 * cz0 : 0);
    const int ncz_loop = live_pair ? cz1 - cz0 : 0;
    // every lane of a warp runs the same number of shuffles: the loop bound is the warp maximum
    int iters = ncz_loop;
    for (int o = 16; o > 0; o >>= 1) iters = max(iters, __shfl_xor_sync(0xffffffffu, iters, o));
    for (int it = 0; it < iters; ++it) {
        const int cz = cz0 + it;
        const bool act = it < ncz_loop;
        Q4<T> acc = zero4<T>();
        if (act) {
            const int zb = 2 * cz;
            double sz = 0.0;
            if constexpr (sizeof(T) == 8) sz = L.d[2][zb] + (zb + 1 < L.nz ? L.d[2][zb + 1] : 0.0);
            for (int kz = 0; kz < 2; ++kz) {
                const int z = zb + kz;
                if (z >= L.nz) break;
                // FP32: the same FP64 quotient, rounded once, from the level's table
                const T wz = sizeof(T) == 4 ? (T)L.rwz[z] : (T)(L.d[2][z] / sz);
                const long i = col.i;
                Q4<T> dg, od, c;
                col.step(dg, od, c);
                if (mine) {
                    const Q4<T> fv = ldq<CG>(f + i);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const T r = dg.a[k] > (T)kEps ? fv.a[k] - (dg.a[k] * c.a[k] + od.a[k]) : (T)0;
                        acc.a[k] += wz * wxy[k] * r;
                    }
                }
            }
        }
        const T ya = acc.a[0] + acc.a[1], yb = acc.a[2] + acc.a[3];
        const T oa = __shfl_xor_sync(0xffffffffu, ya, 1), ob = __shfl_xor_sync(0xffffffffu, yb, 1);
        if (act && xpar == 0) {
            const long ci = (y0 >> 1) + (long)cx * ncy + (long)cz * ncx * ncy;
            fc[ci] = ya + oa;
            fc[ci + 1] = yb + ob;
        }
    }
}

// MINB: register-budget variants as for the Jacobi sweep (1 default, 3 or 4 resident CTAs per SM).
template <typename T, int MINB = 1>
__global__ void __launch_bounds__(256, MINB) resid_restrict_q_kernel(T* __restrict__ fc, const T* __restrict__ v,
                                                                     const T* __restrict__ f, Lvl<T> L, int ncx,
                                                                     int ncy, int ncz, int czc) {
    wp_pdl_enter();
    resid_restrict_q_body<T>(fc, v, f, L, ncx, ncy, ncz, czc, blockIdx.x, blockIdx.y, threadIdx.x);
}

// resid_restrict_q_kernel with its fine planes' streaming loads (the walker's next centre quad and
// f) issued JP_DEPTH - 1 planes ahead into a per-thread cp.async ring (as jacobi_qp_kernel); the
// sums and their order are resid_restrict_q_kernel's.
__global__ void __launch_bounds__(256, 3) resid_restrict_qp_kernel(float* __restrict__ fc,
                                                                   const float* __restrict__ v,
                                                                   const float* __restrict__ f, Lvl<float> L,
                                                                   int ncx, int ncy, int ncz, int czc) {
    wp_pdl_enter();
    extern __shared__ __align__(16) float4 jp_smem[];
    float4 (*ring_v)[256] = reinterpret_cast<float4 (*)[256]>(jp_smem);
    float4 (*ring_f)[256] = reinterpret_cast<float4 (*)[256]>(jp_smem + JP_DEPTH * 256);
    const int tid = threadIdx.x;
    const int nq = L.ny >> 2;
    const long q = (long)blockIdx.x * 256 + tid;
    const int cz0 = blockIdx.y * czc, cz1 = min(cz0 + czc, ncz);
    const long pair = q >> 1;
    const int xpar = (int)(q & 1);
    const bool live_pair = pair < (long)ncx * nq && cz0 < cz1;
    const int cx = live_pair ? (int)(pair / nq) : 0;
    const int y0 = live_pair ? (int)(pair - (long)cx * nq) * 4 : 0;
    const int x0 = 2 * cx;
    const bool two = x0 + 1 < L.nx;
    const bool mine = live_pair && (xpar == 0 || two);
    const int x = mine ? x0 + xpar : x0;
    float wxy[4];
    {
        const double sx = L.d[0][x0] + (two ? L.d[0][x0 + 1] : 0.0);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int y = y0 + k, yb = y & ~1;
            const double sy = L.d[1][yb] + (yb + 1 < L.ny ? L.d[1][yb + 1] : 0.0);
            wxy[k] = mine ? (float)(L.d[1][y] / sy * (L.d[0][x] / sx)) : 0.f;
        }
    }
    // fine planes this lane walks: zs .. ze - 1
    const int zs = 2 * cz0, ze = live_pair ? min(2 * cz1, L.nz) : zs;
    const long sxy = (long)L.nx * L.ny;
    const long ibase = y0 + (long)x * L.ny;
    auto issue = [&](int p) {
        const int slot = (p - zs) % JP_DEPTH;
        if (p < ze) {
            if (p + 1 < L.nz) cp_async16(&ring_v[slot][tid], v + ibase + (long)(p + 1) * sxy);
            cp_async16(&ring_f[slot][tid], f + ibase + (long)p * sxy);
        }
        cp_async_commit();
    };
    if (live_pair)
        for (int p = zs; p < zs + JP_DEPTH - 1; ++p) issue(p);
    QCol<float, float> col(L, v, x, y0, live_pair ? zs : 0);
    const int ncz_loop = live_pair ? cz1 - cz0 : 0;
    int iters = ncz_loop;
    for (int o = 16; o > 0; o >>= 1) iters = max(iters, __shfl_xor_sync(0xffffffffu, iters, o));
    for (int it = 0; it < iters; ++it) {
        const int cz = cz0 + it;
        const bool act = it < ncz_loop;
        Q4<float> acc = zero4<float>();
        if (act) {
            const int zb = 2 * cz;
            for (int kz = 0; kz < 2; ++kz) {
                const int z = zb + kz;
                if (z >= L.nz) break;
                issue(z + JP_DEPTH - 1);
                cp_async_wait<JP_DEPTH - 1>();
                const int slot = (z - zs) % JP_DEPTH;
                const float wz = L.rwz[z];  // (float)(d_z / (d_zb + d_zb+1)), formed in FP64
                const long i = col.i;
                Q4<float> vp = zero4<float>();
                if (z < L.nz - 1) {
                    const float4 t = ring_v[slot][tid];
                    vp = Q4<float>{{t.x, t.y, t.z, t.w}};
                }
                Q4<float> dg, od, c;
                col.step_with(dg, od, c, vp);
                (void)i;
                if (mine) {
                    const float4 tf = ring_f[slot][tid];
                    const Q4<float> fv{{tf.x, tf.y, tf.z, tf.w}};
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const float r = dg.a[k] > (float)kEps ? fv.a[k] - (dg.a[k] * c.a[k] + od.a[k]) : 0.f;
                        acc.a[k] += wz * wxy[k] * r;
                    }
                }
            }
        }
        const float ya = acc.a[0] + acc.a[1], yb = acc.a[2] + acc.a[3];
        const float oa = __shfl_xor_sync(0xffffffffu, ya, 1), ob = __shfl_xor_sync(0xffffffffu, yb, 1);
        if (act && xpar == 0) {
            const long ci = (y0 >> 1) + (long)cx * ncy + (long)cz * ncx * ncy;
            fc[ci] = ya + oa;
            fc[ci + 1] = yb + ob;
        }
    }
    cp_async_wait<0>();
}

// FP64 defect on quads (see defect64_z_kernel): one thread's column of quads of block (bx, by);
// returns its share of ||r||^2.  CG: p through L2 (see ldq).
template <typename TP, bool CG = false>
__device__ __forceinline__ double defect64_q_body(float* __restrict__ r32, const TP* __restrict__ p,
                                                  const float* __restrict__ f, const Lvl<double>& L, double m, int zc,
                                                  int bx, int by, int tid) {
    const int nq = L.ny >> 2;
    const long q = (long)bx * 256 + tid;
    const int z0 = by * zc, z1 = min(z0 + zc, L.nz);
    double s2 = 0.0;
    if (q < (long)L.nx * nq && z0 < z1) {
        const int x = (int)(q / nq), y0 = (int)(q - (long)x * nq) * 4;
        QCol<double, TP, CG> col(L, p, x, y0, z0);
        for (int z = z0; z < z1; ++z) {
            const long i = col.i;
            Q4<double> dg, od, c;
            col.step(dg, od, c);
            const Q4<float> fv = ld4(f + i);
            Q4<float> rr;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double r = dg.a[k] > kEps ? ((double)fv.a[k] - m) - (dg.a[k] * c.a[k] + od.a[k]) : 0.0;
                rr.a[k] = (float)r;
                s2 += r * r;
            }
            if (r32) st4(r32 + i, rr);
        }
    }
    return s2;
}

template <typename TP>
__global__ void __launch_bounds__(256, 2) defect64_q_kernel(float* __restrict__ r32, const TP* __restrict__ p,
                                                         const float* __restrict__ f, Lvl<double> L, double m,
                                                         const double* __restrict__ msum, double* __restrict__ acc,
                                                         int zc) {
    wp_pdl_enter();
    if (msum) m = msum[0] / fmax(msum[1], 1.0);
    double s2 = defect64_q_body<TP>(r32, p, f, L, m, zc, blockIdx.x, blockIdx.y, threadIdx.x);
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < 8; ++k) t += red[k];
        atomicAdd(acc, t);
    }
}

// defect64_q_kernel<double> with the walker's next centre quad of p (FP64) and f issued JP_DEPTH - 1
// planes ahead into a per-thread cp.async ring; the same arithmetic and reduction.
__global__ void __launch_bounds__(256, 2) defect64_qp_kernel(float* __restrict__ r32, const double* __restrict__ p,
                                                             const float* __restrict__ f, Lvl<double> L, double m,
                                                             const double* __restrict__ msum,
                                                             double* __restrict__ acc, int zc) {
    wp_pdl_enter();
    // dynamic shared memory: ring_p (JP_DEPTH x 512 double2) | ring_f (JP_DEPTH x 256 float4)
    extern __shared__ __align__(16) float4 jp_smem[];
    double2 (*ring_p)[512] = reinterpret_cast<double2 (*)[512]>(jp_smem);
    float4 (*ring_f)[256] = reinterpret_cast<float4 (*)[256]>(jp_smem + 2 * JP_DEPTH * 256);
    const int tid = threadIdx.x;
    const int nq = L.ny >> 2;
    const long q = (long)blockIdx.x * 256 + tid;
    const int z0 = blockIdx.y * zc, z1 = min(z0 + zc, L.nz);
    if (msum) m = msum[0] / fmax(msum[1], 1.0);
    double s2 = 0.0;
    if (q < (long)L.nx * nq && z0 < z1) {
        const int x = (int)(q / nq), y0 = (int)(q - (long)x * nq) * 4;
        const long sxy = (long)L.nx * L.ny;
        const long ibase = y0 + (long)x * L.ny;
        auto issue = [&](int pl) {
            const int slot = (pl - z0) % JP_DEPTH;
            if (pl < z1) {
                if (pl + 1 < L.nz) {
                    cp_async16(&ring_p[slot][2 * tid], p + ibase + (long)(pl + 1) * sxy);
                    cp_async16(&ring_p[slot][2 * tid + 1], p + ibase + (long)(pl + 1) * sxy + 2);
                }
                cp_async16(&ring_f[slot][tid], f + ibase + (long)pl * sxy);
            }
            cp_async_commit();
        };
        for (int pl = z0; pl < z0 + JP_DEPTH - 1; ++pl) issue(pl);
        QCol<double, double> col(L, p, x, y0, z0);
        for (int z = z0; z < z1; ++z) {
            issue(z + JP_DEPTH - 1);
            cp_async_wait<JP_DEPTH - 1>();
            const int slot = (z - z0) % JP_DEPTH;
            const long i = col.i;
            Q4<double> vp = zero4<double>();
            if (z < L.nz - 1) {
                const double2 a = ring_p[slot][2 * tid], b = ring_p[slot][2 * tid + 1];
                vp = Q4<double>{{a.x, a.y, b.x, b.y}};
            }
            Q4<double> dg, od, c;
            col.step_with(dg, od, c, vp);
            const float4 tf = ring_f[slot][tid];
            const float fv[4] = {tf.x, tf.y, tf.z, tf.w};
            Q4<float> rr;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double r = dg.a[k] > kEps ? ((double)fv[k] - m) - (dg.a[k] * c.a[k] + od.a[k]) : 0.0;
                rr.a[k] = (float)r;
                s2 += r * r;
            }
            if (r32) st4(r32 + i, rr);
        }
        cp_async_wait<0>();
    }
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < 8; ++k) t += red[k];
        atomicAdd(acc, t);
    }
}

// trilinear prolongation (prolong_tri_add_kernel) on quads: one 128-bit read-modify-write of v
template <typename T, bool CG = false>
__device__ __forceinline__ void prolong_tri_q_body(T* __restrict__ v, const T* __restrict__ vc, int nx, int ny, int nz,
                                                   int ncx, int ncy, int ncz, int bx, int z, int tid) {
    const int nq = ny >> 2;
    const long q = (long)bx * 256 + tid;
    if (q >= (long)nx * nq) return;
    const int x = (int)(q / nq), y0 = (int)(q - (long)x * nq) * 4;
    const int px = x >> 1, pz = z >> 1;
    int qx = (x & 1) ? px + 1 : px - 1, qz = (z & 1) ? pz + 1 : pz - 1;
    if (qx < 0 || qx >= ncx) qx = px;
    if (qz < 0 || qz >= ncz) qz = pz;
    const long sc = (long)ncx * ncy;
    const T a = (T)0.75, b = (T)0.25;
    const long i = y0 + (long)x * ny + (long)z * nx * ny;
    Q4<T> out = ldq<CG>(v + i);
    // the quad's coarse y values along one coarse (x, z) row: cy0 - 1, cy0, cy0 + 1, cy0 + 2, with the
    // wall neighbour repeating the parent (ny % 4 == 0, so ncy = ny / 2 and cy0 = y0 / 2 is even)
    const int cy0 = y0 >> 1;
    struct Row4 {
        T m, a, b, p;
    };
    auto row4 = [&](int xx, int zz) -> Row4 {
        const T* r = vc + cy0 + (long)xx * ncy + zz * sc;
        Row4 o;
        o.a = ld1<CG>(r);
        o.b = ld1<CG>(r + 1);
        o.m = cy0 > 0 ? ld1<CG>(r - 1) : o.a;
        o.p = cy0 + 2 < ncy ? ld1<CG>(r + 2) : o.b;
        return o;
    };
    // parent (P) and neighbour (Q) of cell k of the quad in a row
    auto PQ = [&](const Row4& r, int k, T& P, T& Q) {
        if (k == 0) { P = r.a; Q = r.m; }
        else if (k == 1) { P = r.a; Q = r.b; }
        else if (k == 2) { P = r.b; Q = r.a; }
        else { P = r.b; Q = r.p; }
    };
    if (ncz == 1 && nz == 1) {
        const Row4 r0 = row4(px, 0), r1 = row4(qx, 0);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            T P0, Q0, P1, Q1;
            PQ(r0, k, P0, Q0);
            PQ(r1, k, P1, Q1);
            out.a[k] += a * (a * P0 + b * Q0) + b * (a * P1 + b * Q1);
        }
    } else {
        const Row4 r00 = row4(px, pz), r10 = row4(qx, pz), r01 = row4(px, qz), r11 = row4(qx, qz);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            T P00, Q00, P10, Q10, P01, Q01, P11, Q11;
            PQ(r00, k, P00, Q00);
            PQ(r10, k, P10, Q10);
            PQ(r01, k, P01, Q01);
            PQ(r11, k, P11, Q11);
            const T lo = a * (a * P00 + b * Q00) + b * (a * P10 + b * Q10);
            const T hi = a * (a * P01 + b * Q01) + b * (a * P11 + b * Q11);
            out.a[k] += a * lo + b * hi;
        }
    }
    st4(v + i, out);
}

template <typename T>
__global__ void __launch_bounds__(256) prolong_tri_q_kernel(T* __restrict__ v, const T* __restrict__ vc, int nx, int ny,
                                                            int nz, int ncx, int ncy, int ncz) {
    wp_pdl_enter();
    prolong_tri_q_body<T>(v, vc, nx, ny, nz, ncx, ncy, ncz, blockIdx.x, blockIdx.y, threadIdx.x);
}

#include "wp_mg_fused.cuh"

// cell layout of the y-face fractions: fyc[y + x ny + z nx ny] = ay[y + x (ny+1) + z nx (ny+1)]
__global__ void fyc_kernel(float* __restrict__ fyc, const float* __restrict__ ay, int nx, int ny, long cells) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < cells; t += (long)gridDim.x * blockDim.x) {
        const long row = t / ny;
        const int y = (int)(t - row * ny);
        fyc[t] = ay[y + row * (ny + 1)];
    }
}

// uni[z nx + x] = 1 when every face of row (x, z) that a stencil reads is exactly 1: the lower y
// faces of y >= 1 (fyc), the x faces x and x + 1 and the z faces z and z + 1 that are interior.  One
// warp per row.
__global__ void uniform_rows_kernel(unsigned char* __restrict__ uni, const float* __restrict__ ax,
                                    const float* __restrict__ fyc, const float* __restrict__ az, int nx, int ny,
                                    int nz) {
    const long rows = (long)nx * nz;
    const int lane = threadIdx.x & 31;
    for (long r = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; r < rows; r += ((long)gridDim.x * blockDim.x) >> 5) {
        const int z = (int)(r / nx), x = (int)(r - (long)z * nx);
        const long i = (long)x * ny + (long)z * nx * ny;
        const long ia = (long)x * ny + (long)z * (nx + 1) * ny;
        const long sxy = (long)nx * ny;
        bool ok = true;
        for (int y = lane; y < ny; y += 32) {
            if (y > 0) ok = ok && fyc[i + y] == 1.f;
            if (x > 0) ok = ok && ax[ia + y] == 1.f;
            if (x < nx - 1) ok = ok && ax[ia + ny + y] == 1.f;
            if (z > 0) ok = ok && az[i + y] == 1.f;
            if (z < nz - 1) ok = ok && az[i + sxy + y] == 1.f;
        }
        ok = __all_sync(0xffffffffu, ok);
        if (lane == 0) uni[r] = ok ? 1 : 0;
    }
}

// Fused residual + restriction: each thread walks one fine column, the 2 x 2 children in (y, x)
// are combined with a lane shuffle and a shared-memory exchange, the 2 children in z in registers.
// Coarse value = sum of (dx_x dx_y dx_z / sums) weighted fine residuals (cuRestrict3D.cu:801-970).
template <typename T>
__global__ void __launch_bounds__(256) resid_restrict_z_kernel(T* __restrict__ fc, const T* __restrict__ v,
                                                               const T* __restrict__ f, Lvl<T> L, int ncx, int ncy,
                                                               int ncz, int czc) {
    __shared__ T red[8][16];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int y = blockIdx.x * 32 + tx, x = blockIdx.y * 8 + ty;
    const int cz0 = blockIdx.z * czc, cz1 = min(cz0 + czc, ncz);
    const bool in = y < L.ny && x < L.nx;
    T wxy = 0;
    if (in) {
        const int y0 = y & ~1, x0 = x & ~1;
        const double sy = L.d[1][y0] + (y0 + 1 < L.ny ? L.d[1][y0 + 1] : 0.0);
        const double sx = L.d[0][x0] + (x0 + 1 < L.nx ? L.d[0][x0 + 1] : 0.0);
        wxy = (T)(L.d[1][y] / sy * (L.d[0][x] / sx));
    }
    ZCol<T, T, false> col(L, v, nullptr, 0, 0, in ? x : 0, in ? y : 0, 2 * cz0);
    for (int cz = cz0; cz < cz1; ++cz) {
        T acc = 0;
        const int zb = 2 * cz;
        const double sz = L.d[2][zb] + (zb + 1 < L.nz ? L.d[2][zb + 1] : 0.0);
        for (int k = 0; k < 2; ++k) {
            const int z = zb + k;
            if (z < L.nz && in) {
                const long i = col.i;
                T dg, od, c;
                col.step(dg, od, c);
                const T r = dg > (T)kEps ? f[i] - (dg * c + od) : (T)0;
                acc += (T)(L.d[2][z] / sz) * wxy * r;
            }
        }
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        if ((tx & 1) == 0) red[ty][tx >> 1] = acc;
        __syncthreads();
        if (ty < 4 && tx < 16) {
            const int cy = blockIdx.x * 16 + tx, cx = blockIdx.y * 4 + ty;
            if (cy < ncy && cx < ncx) fc[cy + (long)cx * ncy + (long)cz * ncx * ncy] = red[2 * ty][tx] + red[2 * ty + 1][tx];
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(256) prolong_add_kernel(T* __restrict__ v, const T* __restrict__ vc, int nx, int ny,
                                                          int nz, int ncx, int ncy) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (y >= ny || x >= nx) return;
    v[y + (long)x * ny + (long)z * nx * ny] += vc[(y >> 1) + (long)(x >> 1) * ncy + (long)(z >> 1) * ncx * ncy];
}

// cell-centred trilinear prolongation added into the fine iterate (weights 3/4, 1/4 per axis,
// the missing neighbour at a wall repeats the parent; 2D when nz == 1).  The reference's
// piecewise-constant prolongation (cuProlongate3D.cu:594-617) with its averaging restriction gives
// a coarse correction twice the Galerkin one (R A P = 2 A_coarse) and the V(2,2), omega = 2/3
// cycle stalls and then diverges beyond 64^3; this prolongation restores h-independent convergence.
template <typename T>
__global__ void __launch_bounds__(256) prolong_tri_add_kernel(T* __restrict__ v, const T* __restrict__ vc, int nx, int ny,
                                                              int nz, int ncx, int ncy, int ncz) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (y >= ny || x >= nx) return;
    const int px = x >> 1, py = y >> 1, pz = z >> 1;
    int qx = (x & 1) ? px + 1 : px - 1, qy = (y & 1) ? py + 1 : py - 1, qz = (z & 1) ? pz + 1 : pz - 1;
    if (qx < 0 || qx >= ncx) qx = px;
    if (qy < 0 || qy >= ncy) qy = py;
    if (qz < 0 || qz >= ncz) qz = pz;
    const long sc = (long)ncx * ncy;
    auto C = [&](int xx, int yy, int zz) -> T { return vc[yy + (long)xx * ncy + zz * sc]; };
    T acc;
    const T a = (T)0.75, b = (T)0.25;
    if (ncz == 1 && nz == 1) {
        acc = a * (a * C(px, py, 0) + b * C(px, qy, 0)) + b * (a * C(qx, py, 0) + b * C(qx, qy, 0));
    } else {
        const T lo = a * (a * C(px, py, pz) + b * C(px, qy, pz)) + b * (a * C(qx, py, pz) + b * C(qx, qy, pz));
        const T hi = a * (a * C(px, py, qz) + b * C(px, qy, qz)) + b * (a * C(qx, py, qz) + b * C(qx, qy, qz));
        acc = a * lo + b * hi;
    }
    v[y + (long)x * ny + (long)z * nx * ny] += acc;
}

// ------------------------------------------------------------------ fused coarse cycle
// The V-cycle below a small level (<= kCoarseCells cells) in ONE single-CTA launch: zeroing, sweeps,
// residual restriction, coarsest sweeps and prolongation of every coarse level, with block barriers
// between the steps (the data stay in L2).  At these sizes every separate kernel is a few
// microseconds of launch and ramp for a few thousand cells.  Per cell the arithmetic is that of the
// separate kernels: `row` for the sweeps, and the restriction sums in the order of
// resid_restrict_z_kernel: ((x0,y0) + (x0,y1)) + ((x1,y0) + (x1,y1)), each child (0 + w_z0 r) + w_z1 r.
constexpr int kCoarseMax = 8;
constexpr int kCoarseCells = 4096;

template <typename T>
struct CLev {
    Lvl<T> L;
    T *v, *t, *f;
};
template <typename T>
struct CPack {
    CLev<T> lv[kCoarseMax];
    int n;
};

template <typename T>
__device__ __forceinline__ void cc_sweep(const Lvl<T>& L, T* __restrict__ dst, const T* __restrict__ src,
                                         const T* __restrict__ f, T w) {
    const int nx = L.nx, ny = L.ny, cells = L.nx * L.ny * L.nz;
    for (int i = threadIdx.x; i < cells; i += blockDim.x) {
        const int y = i % ny, x = (i / ny) % nx, z = i / (nx * ny);
        T dg, od, c;
        row<T, T, false>(L, src, nullptr, 0, 0, x, y, z, dg, od, c);
        dst[i] = dg > (T)kEps ? ((T)1 - w) * c + w * (f[i] - od) / dg : (T)0;
    }
}

// the same sweep by one warp (cells <= 32)
template <typename T>
__device__ __forceinline__ void cc_sweep_warp(const Lvl<T>& L, T* __restrict__ dst, const T* __restrict__ src,
                                              const T* __restrict__ f, T w) {
    const int nx = L.nx, ny = L.ny, cells = L.nx * L.ny * L.nz;
    const int i = threadIdx.x;
    if (i < cells) {
        const int y = i % ny, x = (i / ny) % nx, z = i / (nx * ny);
        T dg, od, c;
        row<T, T, false>(L, src, nullptr, 0, 0, x, y, z, dg, od, c);
        dst[i] = dg > (T)kEps ? ((T)1 - w) * c + w * (f[i] - od) / dg : (T)0;
    }
}

template <typename T>
__device__ __forceinline__ void cc_restrict(const Lvl<T>& L, const T* __restrict__ v, const T* __restrict__ f,
                                            T* __restrict__ fc, int ncx, int ncy, int ncz) {
    const int ccells = ncx * ncy * ncz;
    for (int ci = threadIdx.x; ci < ccells; ci += blockDim.x) {
        const int cy = ci % ncy, cx = (ci / ncy) % ncx, cz = ci / (ncx * ncy);
        const int x0 = 2 * cx, y0 = 2 * cy, zb = 2 * cz;
        const double sx = L.d[0][x0] + (x0 + 1 < L.nx ? L.d[0][x0 + 1] : 0.0);
        const double sy = L.d[1][y0] + (y0 + 1 < L.ny ? L.d[1][y0 + 1] : 0.0);
        const double sz = L.d[2][zb] + (zb + 1 < L.nz ? L.d[2][zb + 1] : 0.0);
        T tot[2][2] = {{(T)0, (T)0}, {(T)0, (T)0}};
        for (int xo = 0; xo < 2; ++xo) {
            const int x = x0 + xo;
            if (x >= L.nx) break;
            for (int yo = 0; yo < 2; ++yo) {
                const int y = y0 + yo;
                if (y >= L.ny) break;
                const T wxy = (T)(L.d[1][y] / sy * (L.d[0][x] / sx));
                T acc = 0;
                for (int kz = 0; kz < 2; ++kz) {
                    const int z = zb + kz;
                    if (z >= L.nz) break;
                    T dg, od, c;
                    row<T, T, false>(L, v, nullptr, 0, 0, x, y, z, dg, od, c);
                    const long i = y + (long)x * L.ny + (long)z * L.nx * L.ny;
                    const T r = dg > (T)kEps ? f[i] - (dg * c + od) : (T)0;
                    acc += (T)(L.d[2][z] / sz) * wxy * r;
                }
                tot[xo][yo] = acc;
            }
        }
        fc[ci] = (tot[0][0] + tot[0][1]) + (tot[1][0] + tot[1][1]);
    }
}

template <typename T>
__device__ __forceinline__ void cc_prolong(T* __restrict__ v, const T* __restrict__ vc, int nx, int ny, int nz,
                                           int ncx, int ncy, int ncz, int prolong) {
    const int cells = nx * ny * nz;
    const long sc = (long)ncx * ncy;
    for (int i = threadIdx.x; i < cells; i += blockDim.x) {
        const int y = i % ny, x = (i / ny) % nx, z = i / (nx * ny);
        const int px = x >> 1, py = y >> 1, pz = z >> 1;
        if (prolong != WP_PROLONG_TRILINEAR) {
            v[i] += vc[py + (long)px * ncy + pz * sc];
            continue;
        }
        int qx = (x & 1) ? px + 1 : px - 1, qy = (y & 1) ? py + 1 : py - 1, qz = (z & 1) ? pz + 1 : pz - 1;
        if (qx < 0 || qx >= ncx) qx = px;
        if (qy < 0 || qy >= ncy) qy = py;
        if (qz < 0 || qz >= ncz) qz = pz;
        auto C = [&](int xx, int yy, int zz) -> T { return vc[yy + (long)xx * ncy + zz * sc]; };
        const T a = (T)0.75, b = (T)0.25;
        T acc;
        if (ncz == 1 && nz == 1) {
            acc = a * (a * C(px, py, 0) + b * C(px, qy, 0)) + b * (a * C(qx, py, 0) + b * C(qx, qy, 0));
        } else {
            const T lo = a * (a * C(px, py, pz) + b * C(px, qy, pz)) + b * (a * C(qx, py, pz) + b * C(qx, qy, pz));
            const T hi = a * (a * C(px, py, qz) + b * C(px, qy, qz)) + b * (a * C(qx, py, qz) + b * C(qx, qy, qz));
            acc = a * lo + b * hi;
        }
        v[i] += acc;
    }
}

// V-cycle of the pack's levels; level 0 of the pack has its f and a zeroed v on entry.  Every level's
// v, t and f live in shared memory for the whole cycle (at most kCoarseSmemCells cells in all); the
// face fractions and tables are read through L1.  On exit the finest pack level's v is written to
// the global buffer the host will hold as that level's v after mirroring the nu1 + nu2 swaps.
constexpr int kCoarseSmemCells = 4800;

template <typename T>
__global__ void __launch_bounds__(1024) coarse_cycle_kernel(CPack<T> P, int nu1, int nu2, T w, int citers,
                                                            int prolong) {
    extern __shared__ __align__(16) unsigned char cc_smem[];
    T* base = reinterpret_cast<T*>(cc_smem);
    T* v[kCoarseMax];
    T* t[kCoarseMax];
    T* fs[kCoarseMax];
    {
        int off = 0;
        for (int l = 0; l < P.n; ++l) {
            const int n = P.lv[l].L.nx * P.lv[l].L.ny * P.lv[l].L.nz;
            v[l] = base + off;
            t[l] = base + off + n;
            fs[l] = base + off + 2 * n;
            off += 3 * n;
        }
        const int n0 = P.lv[0].L.nx * P.lv[0].L.ny * P.lv[0].L.nz;
        for (int i = threadIdx.x; i < n0; i += blockDim.x) {
            fs[0][i] = P.lv[0].f[i];
            v[0][i] = (T)0;
        }
        __syncthreads();
    }
    for (int l = 0; l < P.n - 1; ++l) {
        const Lvl<T>& L = P.lv[l].L;
        if (l > 0) {
            const int n = L.nx * L.ny * L.nz;
            for (int i = threadIdx.x; i < n; i += blockDim.x) v[l][i] = (T)0;
            __syncthreads();
        }
        for (int k = 0; k < nu1; ++k) {
            cc_sweep<T>(L, t[l], v[l], fs[l], w);
            __syncthreads();
            T* tmp = v[l];
            v[l] = t[l];
            t[l] = tmp;
        }
        const Lvl<T>& C = P.lv[l + 1].L;
        cc_restrict<T>(L, v[l], fs[l], fs[l + 1], C.nx, C.ny, C.nz);
        __syncthreads();
    }
    {
        const int l = P.n - 1;
        const Lvl<T>& L = P.lv[l].L;
        if (l > 0) {
            const int n = L.nx * L.ny * L.nz;
            for (int i = threadIdx.x; i < n; i += blockDim.x) v[l][i] = (T)0;
            __syncthreads();
        }
        if (L.nx * L.ny * L.nz <= 32) {
            // a coarsest grid of a few cells: one warp iterates alone (warp barriers only)
            if (threadIdx.x < 32) {
                for (int k = 0; k < citers; ++k) {
                    cc_sweep_warp<T>(L, t[l], v[l], fs[l], w);
                    __syncwarp();
                    T* tmp = v[l];
                    v[l] = t[l];
                    t[l] = tmp;
                }
            } else {
                if (citers & 1) {
                    T* tmp = v[l];
                    v[l] = t[l];
                    t[l] = tmp;
                }
            }
            __syncthreads();
        } else {
            for (int k = 0; k < citers; ++k) {
                cc_sweep<T>(L, t[l], v[l], fs[l], w);
                __syncthreads();
                T* tmp = v[l];
                v[l] = t[l];
                t[l] = tmp;
            }
        }
    }
    for (int l = P.n - 2; l >= 0; --l) {
        const Lvl<T>& L = P.lv[l].L;
        const Lvl<T>& C = P.lv[l + 1].L;
        cc_prolong<T>(v[l], v[l + 1], L.nx, L.ny, L.nz, C.nx, C.ny, C.nz, prolong);
        __syncthreads();
        for (int k = 0; k < nu2; ++k) {
            cc_sweep<T>(L, t[l], v[l], fs[l], w);
            __syncthreads();
            T* tmp = v[l];
            v[l] = t[l];
            t[l] = tmp;
        }
    }
    T* out = ((nu1 + nu2) & 1) ? P.lv[0].t : P.lv[0].v;
    const int n0 = P.lv[0].L.nx * P.lv[0].L.ny * P.lv[0].L.nz;
    for (int i = threadIdx.x; i < n0; i += blockDim.x) out[i] = v[0][i];
}

// ---- FP32 coarse cycle on precomputed stencils ------------------------------------------------
// The levels a coarse cycle can hold (cells <= kCoarseCells) keep their stencil per cell, SoA in
// kCcf arrays of `cells` floats: [0..5] the face coefficients (fraction x spacing factor) in the order
// row() applies them (y-, y+, x-, x+, z-, z+), 0 where row() skips the face; [6] row()'s diagonal
// (their sum in that order); [7] the cell's restriction weight (T)(d_z / s_z) * (T)(d_y / s_y *
// (d_x / s_x)) of resid_restrict.  A sweep then needs no index decomposition, no boundary branches
// and no global loads: with v padded by one z plane on either side, the six neighbours are
// i -+ 1, i -+ ny, i -+ nx ny, and a skipped face contributes 0 * (a finite neighbour).
constexpr int kCcf = 8;
constexpr size_t kLeanSmemMax = 226 * 1024;  // dynamic part; the level descriptors are static shared memory

__global__ void cc_coeff_kernel(float* __restrict__ out, Lvl<float> L) {
    const int nx = L.nx, ny = L.ny, nz = L.nz, cells = nx * ny * nz;
    const long sxy = (long)nx * ny;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += gridDim.x * blockDim.x) {
        const int y = i % ny, x = (i / ny) % nx, z = i / (nx * ny);
        const long iax = y + (long)x * ny + (long)z * (nx + 1) * ny;
        const long iay = y + (long)x * (ny + 1) + (long)z * nx * (ny + 1);
        float c[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        float dg = 0.f;
        if (y > 0) { c[0] = L.ay[iay] * L.glo[1][y]; dg += c[0]; }
        if (y < ny - 1) { c[1] = L.ay[iay + 1] * L.ghi[1][y]; dg += c[1]; }
        if (x > 0) { c[2] = L.ax[iax] * L.glo[0][x]; dg += c[2]; }
        if (x < nx - 1) { c[3] = L.ax[iax + ny] * L.ghi[0][x]; dg += c[3]; }
        if (z > 0) { c[4] = L.az[i] * L.glo[2][z]; dg += c[4]; }
        if (z < nz - 1) { c[5] = L.az[i + sxy] * L.ghi[2][z]; dg += c[5]; }
        const int x0 = x & ~1, y0 = y & ~1, zb = z & ~1;
        const double sx = L.d[0][x0] + (x0 + 1 < nx ? L.d[0][x0 + 1] : 0.0);
        const double sy = L.d[1][y0] + (y0 + 1 < ny ? L.d[1][y0 + 1] : 0.0);
        const double sz = L.d[2][zb] + (zb + 1 < nz ? L.d[2][zb + 1] : 0.0);
        const float wxy = (float)(L.d[1][y] / sy * (L.d[0][x] / sx));
        const float wc = (float)(L.d[2][z] / sz) * wxy;
        for (int k = 0; k < 6; ++k) out[(long)k * cells + i] = c[k];
        out[6L * cells + i] = dg;
        out[7L * cells + i] = wc;
    }
}

struct LLev {
    int nx, ny, nz;
    const float* ccf; // kCcf x cells
    float *v, *t;     // global v / t (written for the pack's finest level on exit)
    const float* f;   // global right-hand side (read for the pack's finest level)
};
struct LPack {
    LLev lv[kCoarseMax];
    int n;
};

// shared floats a lean pack needs: per level v and t padded by a z plane on both sides, f, stencils
// (cf_global: the stencils are read from global memory, not staged)
inline long lean_smem_floats(const LPack& P, bool cf_global = false) {
    long s = 0;
    for (int l = 0; l < P.n; ++l) {
        const long c = (long)P.lv[l].nx * P.lv[l].ny * P.lv[l].nz, p = (long)P.lv[l].nx * P.lv[l].ny;
        s += 2 * (c + 2 * p) + c + (cf_global ? 0 : kCcf * c);
    }
    return s;
}

struct LS {
    int nx, ny, nz, cells, nxy;
    float *v, *t, *f; // v, t point past their lower padding plane
    const float* cf;  // kCcf x cells
};

// off = -(sum of the present c_k * v_neighbour) in row()'s order; returns the centre value
__device__ __forceinline__ float lean_off(const LS& S, const float* __restrict__ v, int i, float& od) {
    const float* cf = S.cf;
    const int n = S.cells;
    float o = 0.f;
    o -= cf[i] * v[i - 1];
    o -= cf[n + i] * v[i + 1];
    o -= cf[2 * n + i] * v[i - S.ny];
    o -= cf[3 * n + i] * v[i + S.ny];
    o -= cf[4 * n + i] * v[i - S.nxy];
    o -= cf[5 * n + i] * v[i + S.nxy];
    od = o;
    return v[i];
}

__device__ __forceinline__ void lean_sweep(const LS& S, float* __restrict__ dst, const float* __restrict__ src, float w,
                                           int i0, int step) {
    for (int i = i0; i < S.cells; i += step) {
        float od;
        const float c = lean_off(S, src, i, od);
        const float dg = S.cf[6 * S.cells + i];
        dst[i] = dg > (float)kEps ? (1.f - w) * c + w * (S.f[i] - od) / dg : 0.f;
    }
}

// (x, y, z) of cell i, and the step that adds `step` to i
__device__ __forceinline__ void lean_coord(int i, int nx, int ny, int& x, int& y, int& z) {
    y = i % ny;
    x = (i / ny) % nx;
    z = i / (nx * ny);
}
__device__ __forceinline__ void lean_advance(int& x, int& y, int& z, int bx, int by, int bz, int nx, int ny) {
    y += by;
    if (y >= ny) { y -= ny; ++x; }
    x += bx;
    if (x >= nx) { x -= nx; ++z; }
    z += bz;
}

// residual of the fine level restricted to the coarse right-hand side (cc_restrict's sums and order):
// first every fine cell's residual, by all threads, into the fine level's second buffer (free until
// the post-sweeps write it), then each coarse cell's weighted sum of its children in the same order
__device__ __forceinline__ void lean_restrict(const LS& F, const LS& C) {
    const int B = blockDim.x;
    const float* dgf = F.cf + 6L * F.cells;
    for (int i = threadIdx.x; i < F.cells; i += B) {
        float od;
        const float c = lean_off(F, F.v, i, od);
        const float dg = dgf[i];
        F.t[i] = dg > (float)kEps ? F.f[i] - (dg * c + od) : 0.f;
    }
    __syncthreads();
    int cx, cy, cz;
    lean_coord(threadIdx.x, C.nx, C.ny, cx, cy, cz);
    int bx, by, bz;
    lean_coord(B, C.nx, C.ny, bx, by, bz);
    const float* wcf = F.cf + 7L * F.cells;
    for (int ci = threadIdx.x; ci < C.cells; ci += B) {
        float tot[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
        for (int xo = 0; xo < 2; ++xo) {
            const int x = 2 * cx + xo;
            if (x >= F.nx) break;
            for (int yo = 0; yo < 2; ++yo) {
                const int y = 2 * cy + yo;
                if (y >= F.ny) break;
                float acc = 0.f;
                for (int kz = 0; kz < 2; ++kz) {
                    const int z = 2 * cz + kz;
                    if (z >= F.nz) break;
                    const int i = y + x * F.ny + z * F.nxy;
                    acc += wcf[i] * F.t[i];
                }
                tot[xo][yo] = acc;
            }
        }
        C.f[ci] = (tot[0][0] + tot[0][1]) + (tot[1][0] + tot[1][1]);
        lean_advance(cx, cy, cz, bx, by, bz, C.nx, C.ny);
    }
}

// v += P vc (cc_prolong's arithmetic)
__device__ __forceinline__ void lean_prolong(const LS& F, const LS& C, int prolong) {
    const int B = blockDim.x;
    int x, y, z;
    lean_coord(threadIdx.x, F.nx, F.ny, x, y, z);
    int bx, by, bz;
    lean_coord(B, F.nx, F.ny, bx, by, bz);
    const int ncx = C.nx, ncy = C.ny, ncz = C.nz;
    const float* vc = C.v;
    for (int i = threadIdx.x; i < F.cells; i += B) {
        const int px = x >> 1, py = y >> 1, pz = z >> 1;
        if (prolong != WP_PROLONG_TRILINEAR) {
            F.v[i] += vc[py + px * ncy + pz * C.nxy];
        } else {
            int qx = (x & 1) ? px + 1 : px - 1, qy = (y & 1) ? py + 1 : py - 1, qz = (z & 1) ? pz + 1 : pz - 1;
            if (qx < 0 || qx >= ncx) qx = px;
            if (qy < 0 || qy >= ncy) qy = py;
            if (qz < 0 || qz >= ncz) qz = pz;
            auto Cv = [&](int xx, int yy, int zz) -> float { return vc[yy + xx * ncy + zz * C.nxy]; };
            const float a = 0.75f, b = 0.25f;
            float acc;
            if (ncz == 1 && F.nz == 1) {
                acc = a * (a * Cv(px, py, 0) + b * Cv(px, qy, 0)) + b * (a * Cv(qx, py, 0) + b * Cv(qx, qy, 0));
            } else {
                const float lo =
                    a * (a * Cv(px, py, pz) + b * Cv(px, qy, pz)) + b * (a * Cv(qx, py, pz) + b * Cv(qx, qy, pz));
                const float hi =
                    a * (a * Cv(px, py, qz) + b * Cv(px, qy, qz)) + b * (a * Cv(qx, py, qz) + b * Cv(qx, qy, qz));
                acc = a * lo + b * hi;
            }
            F.v[i] += acc;
        }
        lean_advance(x, y, z, bx, by, bz, F.nx, F.ny);
    }
}

// coarse_cycle_kernel<float> on the precomputed stencils, everything in shared memory: the same
// cycle, the same arithmetic per cell, the same output buffer.  The pack's stencils are one
// contiguous global block (the levels of at most kCoarseCells cells are allocated together, in
// level order), copied with 128-bit loads that keep many requests in flight; the level
// descriptors live in shared memory (no local-memory arrays), and thread 0 writes back the
// ping-pong state of a level after its sweeps (every thread swaps its own copy in lockstep).
// The body, run by one 1024-thread CTA (also as the coarse phase of mid_cycle_kernel, whose other
// CTAs wrote the pack's right-hand side in the same grid: hence the L2 load of f).
// CFG: the stencils stay in global memory (read through L1) and only v, t, f are staged, for a CTA
// that keeps its shared memory small (the persistent batch kernel).
template <bool CFG = false>
__device__ __forceinline__ void lean_cycle(const LPack& P, int nu1, int nu2, float w, int citers, int prolong,
                                           float* lean_smem) {
    __shared__ LS S[kCoarseMax];
    const int tid = threadIdx.x, B = blockDim.x;
    long cf_floats = 0;
    if (!CFG)
        for (int l = 0; l < P.n; ++l) cf_floats += (long)kCcf * P.lv[l].nx * P.lv[l].ny * P.lv[l].nz;
    if (tid == 0) {
        long cfo = 0, off = cf_floats;
        for (int l = 0; l < P.n; ++l) {
            LS& q = S[l];
            q.nx = P.lv[l].nx;
            q.ny = P.lv[l].ny;
            q.nz = P.lv[l].nz;
            q.nxy = q.nx * q.ny;
            q.cells = q.nxy * q.nz;
            q.cf = CFG ? P.lv[l].ccf : lean_smem + cfo;
            cfo += (long)kCcf * q.cells;
            q.v = lean_smem + off + q.nxy;
            off += q.cells + 2 * q.nxy;
            q.t = lean_smem + off + q.nxy;
            off += q.cells + 2 * q.nxy;
            q.f = lean_smem + off;
            off += q.cells;
        }
    }
    if (!CFG) {
        // stencils: 16-byte asynchronous copies (every level's block is a multiple of 16 bytes), all in
        // flight at once while the buffers are cleared below, waited for before the first sweep
        const char* g = reinterpret_cast<const char*>(P.lv[0].ccf);
        char* d = reinterpret_cast<char*>(lean_smem);
        const int n16 = (int)(cf_floats / 4);
        for (int i = tid; i < n16; i += B) cp_async16(d + 16L * i, g + 16L * i);
        cp_async_commit();
    }
    __syncthreads();
    for (int l = 0; l < P.n; ++l) {
        // padding planes stay zero; level 0 starts from v = 0 and the global f
        const LS q = S[l];
        for (int i = tid; i < q.cells + 2 * q.nxy; i += B) {
            q.v[i - q.nxy] = 0.f;
            q.t[i - q.nxy] = 0.f;
        }
        if (l == 0)
            for (int i = tid; i < q.cells; i += B) q.f[i] = __ldcg(P.lv[0].f + i);
    }
    cp_async_wait<0>();
    __syncthreads();
    for (int l = 0; l < P.n - 1; ++l) {
        LS L = S[l];
        if (l > 0) {
            for (int i = tid; i < L.cells; i += B) L.v[i] = 0.f;
            __syncthreads();
        }
        for (int k = 0; k < nu1; ++k) {
            lean_sweep(L, L.t, L.v, w, tid, B);
            __syncthreads();
            float* tmp = L.v;
            L.v = L.t;
            L.t = tmp;
        }
        lean_restrict(L, S[l + 1]);
        if (tid == 0) {
            S[l].v = L.v;
            S[l].t = L.t;
        }
        __syncthreads();
    }
    {
        LS L = S[P.n - 1];
        if (P.n > 1) {
            for (int i = tid; i < L.cells; i += B) L.v[i] = 0.f;
            __syncthreads();
        }
        if (L.cells <= 32) {
            // a coarsest grid of at most 32 cells: one warp iterates alone, a cell per lane in
            // registers, the neighbours' values by shuffle -- lean_sweep's arithmetic and order, the
            // padding planes (indices outside the level) reading 0.  The result goes to the buffer the
            // swaps of citers sweeps would leave it in.  A single cell has no interior face: its
            // diagonal is 0 and the buffers already hold the 0 every sweep would write.
            if (tid < 32 && L.cells > 1) {
                const int n = L.cells, i = tid;
                const bool own = i < n;
                const int off[6] = {-1, 1, -L.ny, L.ny, -L.nxy, L.nxy};
                float cfk[6], dg = 0.f, fv = 0.f, v = 0.f;
#pragma unroll
                for (int k = 0; k < 6; ++k) cfk[k] = own ? L.cf[k * n + i] : 0.f;
                if (own) {
                    dg = L.cf[6 * n + i];
                    fv = L.f[i];
                    v = L.v[i];
                }
                for (int it = 0; it < citers; ++it) {
                    float o = 0.f;
#pragma unroll
                    for (int k = 0; k < 6; ++k) {
                        const int j = i + off[k];
                        const float vj = __shfl_sync(0xffffffffu, v, j & 31);
                        o -= cfk[k] * ((j >= 0 && j < n) ? vj : 0.f);
                    }
                    const float nv = dg > (float)kEps ? (1.f - w) * v + w * (fv - o) / dg : 0.f;
                    v = own ? nv : v;
                }
                if (own) ((citers & 1) ? L.t : L.v)[i] = v;
            }
            if (citers & 1) {
                float* tmp = L.v;
                L.v = L.t;
                L.t = tmp;
            }
        } else {
            for (int k = 0; k < citers; ++k) {
                lean_sweep(L, L.t, L.v, w, tid, B);
                __syncthreads();
                float* tmp = L.v;
                L.v = L.t;
                L.t = tmp;
            }
        }
        if (tid == 0) {
            S[P.n - 1].v = L.v;
            S[P.n - 1].t = L.t;
        }
        __syncthreads();
    }
    for (int l = P.n - 2; l >= 0; --l) {
        LS L = S[l];
        lean_prolong(L, S[l + 1], prolong);
        __syncthreads();
        for (int k = 0; k < nu2; ++k) {
            lean_sweep(L, L.t, L.v, w, tid, B);
            __syncthreads();
            float* tmp = L.v;
            L.v = L.t;
            L.t = tmp;
        }
        if (tid == 0) {
            S[l].v = L.v;
            S[l].t = L.t;
        }
        __syncthreads();
    }
    float* out = ((nu1 + nu2) & 1) ? P.lv[0].t : P.lv[0].v;
    const float* v0 = S[0].v;
    for (int i = tid; i < S[0].cells; i += B) out[i] = v0[i];
}

__global__ void __launch_bounds__(1024) coarse_cycle_lean_kernel(LPack P, int nu1, int nu2, float w, int citers,
                                                                 int prolong) {
    wp_pdl_enter();
    extern __shared__ __align__(16) float lean_smem[];
    lean_cycle(P, nu1, nu2, w, citers, prolong, lean_smem);
}

// ---- persistent cycle below the finest level --------------------------------------------------
// Levels 1 .. k of a V-cycle are small (at 256^3: 128^3, 64^3, 32^3), L2-resident and latency bound:
// as separate launches each sweep costs a launch, a ramp and a tail.  mid_cycle_kernel runs the whole
// cycle below the finest level in one cooperative launch (one 1024-thread CTA per SM, all resident):
// a list of phases -- first sweep from zero, sweeps, residual restriction, trilinear prolongation
// and the single-CTA coarse cycle -- separated by grid barriers.  A phase runs the quad kernels'
// bodies (the same arithmetic per cell) on virtual 256-thread blocks, four per CTA, with every load
// of data written earlier in the grid taken through L2 (CG).  The host mirrors the ping-pong swaps and
// writes each phase's buffers into the list.
enum { MP_SWEEP0 = 0, MP_SWEEP = 1, MP_RESTRICT = 2, MP_PROLONG = 3, MP_COARSE = 4 };
constexpr int kMidLevels = 6;
constexpr int kMidPhases = 48;

struct MidPhase {
    int type, level, zc, gx, gy;
    float* dst;        // sweep output / restricted right-hand side / prolongation target
    const float* src;  // sweep input / fine iterate of the restriction / coarse correction
    const float* f;    // right-hand side of the level
};
struct MidPack {
    Lvl<float> L[kMidLevels];
    MidPhase ph[kMidPhases];
    LPack coarse;
    int nph, nu1, nu2, citers, prolong;
    float w;
    unsigned* bar;  // [arrivals, generation]
    int* err;
    int withhold;             // test only: 1 = the last CTA skips the first barrier
    unsigned long long lim;   // wait limit of the barriers, ns
};
static_assert(sizeof(MidPack) < 32000, "kernel parameters are limited to 32 KB");

// Grid-wide barrier of a cooperative launch (all CTAs resident): arrivals counted on bar[0], the last
// one resets it and advances the generation bar[1], the others wait for that (bounded: after
// lim ns the error flag is raised and false returned, and the grid leaves the kernel).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned nblocks, int* err, unsigned long long lim) {
    __syncthreads();
    int ok = 1;
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) + 1u == nblocks) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const unsigned long long t0 = wptc::globaltimer();
            while (*gen == g) {
                if (wptc::globaltimer() - t0 > lim) {
                    atomicOr(err, 2);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
    }
    return __syncthreads_and(ok) != 0;
}

__global__ void __launch_bounds__(1024, 1) mid_cycle_kernel(MidPack P) {
    extern __shared__ __align__(16) float lean_smem[];
    const int sub = threadIdx.x >> 8, tid = threadIdx.x & 255;
    const int vstep = gridDim.x * 4;
    for (int k = 0; k < P.nph; ++k) {
        const MidPhase& ph = P.ph[k];
        if (ph.type == MP_COARSE) {
            if (blockIdx.x == 0) lean_cycle(P.coarse, P.nu1, P.nu2, P.w, P.citers, P.prolong, lean_smem);
        } else {
            const Lvl<float>& L = P.L[ph.level];
            const int nv = ph.gx * ph.gy;
            for (int vb = blockIdx.x * 4 + sub; vb < nv; vb += vstep) {
                const int bx = vb % ph.gx, by = vb / ph.gx;
                if (ph.type == MP_SWEEP0) {
                    jacobi0_q_body<float, true>(ph.dst, ph.f, L, P.w, ph.zc, bx, by, tid);
                } else if (ph.type == MP_SWEEP) {
                    jacobi_q_body<float, false, true>(ph.dst, ph.src, ph.f, L, P.w, ph.zc, nullptr, bx, by, tid);
                } else if (ph.type == MP_RESTRICT) {
                    const Lvl<float>& C = P.L[ph.level + 1];
                    resid_restrict_q_body<float, true>(ph.dst, ph.src, ph.f, L, C.nx, C.ny, C.nz, ph.zc, bx, by,
                                                        tid);
                } else {
                    const Lvl<float>& C = P.L[ph.level + 1];
                    prolong_tri_q_body<float, true>(ph.dst, ph.src, L.nx, L.ny, L.nz, C.nx, C.ny, C.nz, bx, by,
                                                     tid);
                }
            }
        }
        if (k == 0 && P.withhold && blockIdx.x == gridDim.x - 1) return;
        if (k + 1 < P.nph && !grid_barrier(P.bar, gridDim.x, P.err, P.lim)) return;
    }
}

// coarse f = spacing-weighted average of the fine residuals of the (up to 8) children
template <typename T>
__global__ void __launch_bounds__(256) resid_restrict_kernel(T* __restrict__ fc, const T* __restrict__ v,
                                                             const T* __restrict__ f, Lvl<T> L, int ncx, int ncy,
                                                             int ncz) {
    const int cy = blockIdx.x * 32 + threadIdx.x, cx = blockIdx.y * 8 + threadIdx.y, cz = blockIdx.z;
    if (cy >= ncy || cx >= ncx) return;
    T acc = 0;
    double wsum[3];
    int cnt[3];
    const int c3[3] = {cx, cy, cz};
    const int n3[3] = {L.nx, L.ny, L.nz};
    for (int a = 0; a < 3; ++a) {
        const int i0 = 2 * c3[a];
        cnt[a] = (i0 + 1 < n3[a]) ? 2 : 1;
        wsum[a] = L.d[a][i0] + (cnt[a] == 2 ? L.d[a][i0 + 1] : 0.0);
    }
    for (int cz2 = 0; cz2 < cnt[2]; ++cz2)
        for (int cx2 = 0; cx2 < cnt[0]; ++cx2)
            for (int cy2 = 0; cy2 < cnt[1]; ++cy2) {
                const int x = 2 * cx + cx2, y = 2 * cy + cy2, z = 2 * cz + cz2;
                T dg, od, c;
                row<T, T, false>(L, v, nullptr, 0, 0, x, y, z, dg, od, c);
                const long i = y + (long)x * L.ny + (long)z * L.nx * L.ny;
                const T r = dg > (T)kEps ? f[i] - (dg * c + od) : (T)0;
                const T wgt = (T)(L.d[0][x] / wsum[0] * (L.d[1][y] / wsum[1]) * (L.d[2][z] / wsum[2]));
                acc += wgt * r;
            }
    fc[cy + (long)cx * ncy + (long)cz * ncx * ncy] = acc;
}

// coarsest level: `iters` weighted-Jacobi sweeps of the whole (small) grid inside one CTA
template <typename T>
__global__ void __launch_bounds__(1024) coarsest_kernel(T* __restrict__ v, const T* __restrict__ f, Lvl<T> L, T w,
                                                        int iters) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* b0 = reinterpret_cast<T*>(smem_raw);
    const int n = L.nx * L.ny * L.nz;
    T* b1 = b0 + n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) b0[i] = v[i];
    __syncthreads();
    T* cur = b0;
    T* nxt = b1;
    for (int it = 0; it < iters; ++it) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int y = i % L.ny, x = (i / L.ny) % L.nx, z = i / (L.ny * L.nx);
            T dg, od, c;
            row<T, T, false>(L, cur, nullptr, 0, 0, x, y, z, dg, od, c);
            nxt[i] = dg > (T)kEps ? ((T)1 - w) * c + w * (f[i] - od) / dg : (T)0;
        }
        __syncthreads();
        T* t = cur; cur = nxt; nxt = t;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) v[i] = cur[i];
}

// FP64 defect r = (f - m) - A p of an iterate p (float or double) on active cells (diag > eps),
// where m is the mean of f over the active cells (0 keeps the reference's plain f - A p);
// optional FP32 copy of r; adds sum r^2 into acc[0]
template <typename TP>
__global__ void __launch_bounds__(256) defect64_kernel(float* __restrict__ r32, const TP* __restrict__ p,
                                                       const float* __restrict__ f, Lvl<double> L, double m,
                                                       double* __restrict__ acc) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    double r = 0.0;
    if (y < L.ny && x < L.nx) {
        double dg, od, c;
        row<double, TP, false>(L, p, nullptr, 0, 0, x, y, z, dg, od, c);
        const long i = y + (long)x * L.ny + (long)z * L.nx * L.ny;
        r = dg > kEps ? ((double)f[i] - m) - (dg * c + od) : 0.0;
        if (r32) r32[i] = (float)r;
    }
    double s = r * r;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double red[8];
    const int lane = threadIdx.x + 32 * threadIdx.y;
    if ((lane & 31) == 0) red[lane >> 5] = s;
    __syncthreads();
    if (lane == 0) {
        double t = 0.0;
        for (int k = 0; k < 8; ++k) t += red[k];
        atomicAdd(acc, t);
    }
}

// sum of f and number of cells over the active cells (diag > eps) into acc[0], acc[1].  With zero-flux
// walls the operator's null space is the constant on the active cells, so a right-hand side stored
// in FP32 carries an incompatible constant part of FP32 rounding size that floors the residual
// (about 2e-10 relative at 64^3); the tolerance-driven solve removes that mean in FP64.
template <typename TP>
__global__ void __launch_bounds__(256) defect64_z_kernel(float* __restrict__ r32, const TP* __restrict__ p,
                                                         const float* __restrict__ f, Lvl<double> L, double m,
                                                         const double* __restrict__ msum, double* __restrict__ acc,
                                                         int zc) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y;
    const int z0 = blockIdx.z * zc, z1 = min(z0 + zc, L.nz);
    if (msum) m = msum[0] / fmax(msum[1], 1.0);  // mean of f over the active cells, computed on the device
    double s2 = 0.0;
    if (y < L.ny && x < L.nx && z0 < z1) {
        ZCol<double, TP, false> col(L, p, nullptr, 0, 0, x, y, z0);
        for (int z = z0; z < z1; ++z) {
            const long i = col.i;
            double dg, od, c;
            col.step(dg, od, c);
            const double r = dg > kEps ? ((double)f[i] - m) - (dg * c + od) : 0.0;
            if (r32) r32[i] = (float)r;
            s2 += r * r;
        }
    }
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    __shared__ double red[8];
    const int lane = threadIdx.x + 32 * threadIdx.y;
    if ((lane & 31) == 0) red[lane >> 5] = s2;
    __syncthreads();
    if (lane == 0) {
        double t = 0.0;
        for (int k = 0; k < 8; ++k) t += red[k];
        atomicAdd(acc, t);
    }
}

__global__ void __launch_bounds__(256) active_sum_kernel(const float* __restrict__ f, Lvl<double> L,
                                                         double* __restrict__ acc) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    double sf = 0.0, cnt = 0.0;
    if (y < L.ny && x < L.nx) {
        double dg, od, c;
        row<double, float, false>(L, f, nullptr, 0, 0, x, y, z, dg, od, c);
        if (dg > kEps) { sf = (double)c; cnt = 1.0; }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sf += __shfl_xor_sync(0xffffffffu, sf, o);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    __shared__ double red[2][8];
    const int lane = threadIdx.x + 32 * threadIdx.y;
    if ((lane & 31) == 0) { red[0][lane >> 5] = sf; red[1][lane >> 5] = cnt; }
    __syncthreads();
    if (lane == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < 8; ++k) { a += red[0][k]; b += red[1][k]; }
        atomicAdd(acc, a);
        atomicAdd(acc + 1, b);
    }
}

// active_sum_kernel on quads: each thread walks a z-chunk of a quad column with the FP64 walker
// (the same diagonal as row()), sums f and the count of active cells, one atomic pair per CTA
__global__ void __launch_bounds__(256) active_sum_q_kernel(const float* __restrict__ f, Lvl<double> L,
                                                           double* __restrict__ acc, int zc) {
    const int nq = L.ny >> 2;
    const long q = (long)blockIdx.x * 256 + threadIdx.x;
    const int z0 = blockIdx.y * zc, z1 = min(z0 + zc, L.nz);
    double sf = 0.0, cnt = 0.0;
    if (q < (long)L.nx * nq && z0 < z1) {
        const int x = (int)(q / nq), y0 = (int)(q - (long)x * nq) * 4;
        QCol<double, float> col(L, f, x, y0, z0);
        for (int z = z0; z < z1; ++z) {
            Q4<double> dg, od, c;
            col.step(dg, od, c);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (dg.a[k] > kEps) { sf += c.a[k]; cnt += 1.0; }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sf += __shfl_xor_sync(0xffffffffu, sf, o);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    __shared__ double red[2][8];
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = sf; red[1][threadIdx.x >> 5] = cnt; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < 8; ++k) { a += red[0][k]; b += red[1][k]; }
        atomicAdd(acc, a);
        atomicAdd(acc + 1, b);
    }
}

// FP64 right-hand side of the compatible problem: f - m on active cells, 0 elsewhere
__global__ void __launch_bounds__(256) rhs64_kernel(double* __restrict__ out, const float* __restrict__ f, Lvl<double> L,
                                                    double m) {
    const int y = blockIdx.x * 32 + threadIdx.x, x = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (y >= L.ny || x >= L.nx) return;
    double dg, od, c;
    row<double, float, false>(L, f, nullptr, 0, 0, x, y, z, dg, od, c);
    out[y + (long)x * L.ny + (long)z * L.nx * L.ny] = dg > kEps ? (double)c - m : 0.0;
}

template <typename TS>
__global__ void __launch_bounds__(256) sumsq_kernel(const TS* __restrict__ a, long n, double* __restrict__ acc) {
    double s = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double v = (double)a[i];
        s += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
        atomicAdd(acc, t);
    }
}

__global__ void add_correction_kernel(double* __restrict__ p, const float* __restrict__ e, long n) {
    wp_pdl_enter();
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) p[i] += (double)e[i];
}

template <typename TD, typename TS>
__global__ void convert_kernel(TD* __restrict__ d, const TS* __restrict__ s, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) d[i] = (TD)s[i];
}

// ------------------------------------------------------------------ index-sparse cycle
// CuMultigridFrac3D::Solve_index (cuMultigridFrac3D.cu:347-420) sweeps, restricts and prolongs only
// the cells that CuBoundSelector::SelectByFrac (cuBoundSelector.cu:4-32) selects -- those with a
// face fraction >= 1e-12 -- from per-level index lists built by a prefix sum (InitIndex, :189-229).
// Here the unit of the list is a segment: 32 consecutive cells along y of one (x, z) row that hold
// at least one selected cell, with the lane mask of the selected ones.  One warp per segment keeps
// every load a 128-byte row piece (the y-fastest layout), solid rows cost nothing, and the mask
// carries the per-cell selection to the kernels.  Segments are stored in memory order.
constexpr int kIxBlock = 1024;  // segments per CTA of the list build

// bit k of mask[s] = cell y0 + k of segment s is selected (the fractions compared in FP64, as the
// reference compares them in its DTYPE); cells counts the selected cells
__global__ void __launch_bounds__(256) index_mask_kernel(unsigned* __restrict__ mask,
                                                         unsigned long long* __restrict__ cells, Lvl<float> L,
                                                         int nsy, long nseg) {
    const long s = ((long)blockIdx.x * 256 + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= nseg) return;  // uniform across the warp
    const long row = s / nsy;
    const int x = (int)(row % L.nx), z = (int)(row / L.nx), y = (int)(s - row * nsy) * 32 + lane;
    bool on = false;
    if (y < L.ny) {
        const long sl = (long)L.nx * L.ny, i = y + (long)x * L.ny + z * sl;
        const long iax = y + (long)x * L.ny + (long)z * (L.nx + 1) * L.ny;
        const long iay = y + (long)x * (L.ny + 1) + (long)z * L.nx * (L.ny + 1);
        on = !((double)L.ax[iax] < kEps && (double)L.ax[iax + L.ny] < kEps && (double)L.ay[iay] < kEps &&
               (double)L.ay[iay + 1] < kEps && (double)L.az[i] < kEps && (double)L.az[i + sl] < kEps);
    }
    const unsigned m = __ballot_sync(0xffffffffu, on);
    if (lane == 0) {
        mask[s] = m;
        if (m) atomicAdd(cells, (unsigned long long)__popc(m));
    }
}

// segments with a selected cell per CTA of kIxBlock segments
__global__ void __launch_bounds__(kIxBlock) index_count_kernel(const unsigned* __restrict__ mask, long nseg,
                                                               int* __restrict__ bcount) {
    const long s = (long)blockIdx.x * kIxBlock + threadIdx.x;
    const int c = __syncthreads_count(s < nseg && mask[s] != 0u);
    if (threadIdx.x == 0) bcount[blockIdx.x] = c;
}

// exclusive scan of the per-CTA counts in place, in one CTA; *total = the listed segments
__global__ void __launch_bounds__(1024) index_scan_kernel(int* __restrict__ bcount, int nb,
                                                          long long* __restrict__ total) {
    __shared__ int part[1024];
    const int t = threadIdx.x;
    const int per = (nb + 1023) / 1024;
    const int b0 = min(t * per, nb), b1 = min(b0 + per, nb);
    int sum = 0;
    for (int b = b0; b < b1; ++b) sum += bcount[b];
    part[t] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = part[t] - sum;
    for (int b = b0; b < b1; ++b) {
        const int c = bcount[b];
        bcount[b] = run;
        run += c;
    }
    if (t == 1023) *total = part[1023];
}

// writes the listed segments {x, z, y0, mask} at the scanned offsets, in memory order
__global__ void __launch_bounds__(kIxBlock) index_scatter_kernel(const unsigned* __restrict__ mask, long nseg,
                                                                 const int* __restrict__ boff, int4* __restrict__ seg,
                                                                 int nsy, int nx) {
    __shared__ int wbase[kIxBlock / 32];
    const long s = (long)blockIdx.x * kIxBlock + threadIdx.x;
    const unsigned m = s < nseg ? mask[s] : 0u;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned b = __ballot_sync(0xffffffffu, m != 0u);
    if (lane == 0) wbase[wid] = __popc(b);
    __syncthreads();
    if (wid == 0) {
        const int own = wbase[lane];
        int v = own;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
        }
        wbase[lane] = v - own;
    }
    __syncthreads();
    if (m) {
        const long row = s / nsy;
        const int pos = boff[blockIdx.x] + wbase[wid] + __popc(b & ((1u << lane) - 1u));
        seg[pos] = make_int4((int)(row % nx), (int)(row / nx), (int)(s - row * nsy) * 32, (int)m);
    }
}

// the cell this lane owns: segment (blockIdx.x * 8 + warp), lane k = cell y0 + k; false when the
// segment does not exist or does not select the cell.  All lanes load the same 16-byte entry.
__device__ __forceinline__ bool index_cell(const int4* __restrict__ seg, long nseg, int& x, int& y, int& z) {
    const long s = ((long)blockIdx.x * 256 + threadIdx.x) >> 5;
    if (s >= nseg) return false;
    const int4 g = seg[s];
    const int lane = threadIdx.x & 31;
    if (!(((unsigned)g.w >> lane) & 1u)) return false;
    x = g.x;
    z = g.y;
    y = g.z + lane;
    return true;
}

// cuWjFrac3D_n with an index (cuWeightedJacobi3D.cu:2821-2897): listed cells only; the others keep
// their value in both buffers
template <typename T>
__global__ void __launch_bounds__(256) jacobi_ix_kernel(T* __restrict__ dst, const T* __restrict__ src,
                                                        const T* __restrict__ f, Lvl<T> L, T w,
                                                        const int4* __restrict__ seg, long nseg) {
    wp_pdl_enter();
    int x, y, z;
    if (!index_cell(seg, nseg, x, y, z)) return;
    T dg, od, c;
    row<T, T, false>(L, src, nullptr, 0, 0, x, y, z, dg, od, c);
    const long i = y + (long)x * L.ny + (long)z * L.nx * L.ny;
    dst[i] = dg > (T)kEps ? ((T)1 - w) * c + w * (f[i] - od) / dg : (T)0;
}

// the first sweep of a coarse level from v = 0 (the reference clears the level, then sweeps): the
// same value as jacobi_ix_kernel on a zero iterate without reading it
template <typename T>
__global__ void __launch_bounds__(256) jacobi0_ix_kernel(T* __restrict__ dst, const T* __restrict__ f, Lvl<T> L,
                                                         T w, const int4* __restrict__ seg, long nseg) {
    wp_pdl_enter();
    int x, y, z;
    if (!index_cell(seg, nseg, x, y, z)) return;
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const long sxy = (long)nx * ny, i = y + (long)x * ny + (long)z * sxy;
    const long iax = y + (long)x * ny + (long)z * (nx + 1) * ny, iay = y + (long)x * (ny + 1) + (long)z * nx * (ny + 1);
    T dg = 0;
    if (y > 0) dg += (T)L.ay[iay] * L.glo[1][y];
    if (y < ny - 1) dg += (T)L.ay[iay + 1] * L.ghi[1][y];
    if (x > 0) dg += (T)L.ax[iax] * L.glo[0][x];
    if (x < nx - 1) dg += (T)L.ax[iax + ny] * L.ghi[0][x];
    if (z > 0) dg += (T)L.az[i] * L.glo[2][z];
    if (z < nz - 1) dg += (T)L.az[i + sxy] * L.ghi[2][z];
    dst[i] = dg > (T)kEps ? w * f[i] / dg : (T)0;
}

// cuWjGetFracRes_3d_n with an index (cuWeightedJacobi3D.cu:3013-3090): the residual of the listed
// cells into the workspace shared by all levels
template <typename T>
__global__ void __launch_bounds__(256) resid_ix_kernel(T* __restrict__ r, const T* __restrict__ v,
                                                       const T* __restrict__ f, Lvl<T> L,
                                                       const int4* __restrict__ seg, long nseg) {
    wp_pdl_enter();
    int x, y, z;
    if (!index_cell(seg, nseg, x, y, z)) return;
    T dg, od, c;
    row<T, T, false>(L, v, nullptr, 0, 0, x, y, z, dg, od, c);
    const long i = y + (long)x * L.ny + (long)z * L.nx * L.ny;
    r[i] = dg > (T)kEps ? f[i] - (dg * c + od) : (T)0;
}

// cuRestrict3D_p1_dx_whole (cuRestrict3D.cu:1146-1193): each listed coarse cell averages the
// workspace over its (up to 8) children with the fine spacings as weights -- every child, listed
// or not, as the reference reads them; the term order is the reference's
template <typename T>
__global__ void __launch_bounds__(256) restrict_ix_kernel(T* __restrict__ fc, const T* __restrict__ r, Lvl<T> L,
                                                          int ncx, int ncy, const int4* __restrict__ cseg,
                                                          long ncseg) {
    wp_pdl_enter();
    int cx, cy, cz;
    if (!index_cell(cseg, ncseg, cx, cy, cz)) return;
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const int xs = 2 * cx, ys = 2 * cy, zs = 2 * cz;
    const bool hx = xs < nx - 1, hy = ys < ny - 1, hz = zs < nz - 1;
    const T wxl = (T)L.d[0][xs], wyl = (T)L.d[1][ys], wzl = (T)L.d[2][zs];
    const T wxr = hx ? (T)L.d[0][xs + 1] : (T)0, wyr = hy ? (T)L.d[1][ys + 1] : (T)0;
    const T wzr = hz ? (T)L.d[2][zs + 1] : (T)0;
    const long ox = hx ? ny : 0, oy = hy ? 1 : 0, oz = hz ? (long)nx * ny : 0;
    long s0 = ys + (long)xs * ny + (long)zs * nx * ny;
    T val = wxl * wyl * wzl * r[s0];
    val += wxl * wyr * wzl * r[s0 + oy];
    val += wxr * wyl * wzl * r[s0 + ox];
    val += wxr * wyr * wzl * r[s0 + oy + ox];
    s0 += oz;
    val += wxl * wyl * wzr * r[s0];
    val += wxl * wyr * wzr * r[s0 + oy];
    val += wxr * wyl * wzr * r[s0 + ox];
    val += wxr * wyr * wzr * r[s0 + oy + ox];
    fc[cy + (long)cx * ncy + (long)cz * ncx * ncy] = val / ((wxl + wxr) * (wyl + wyr) * (wzl + wzr));
}

// cuProlongate3D_p1_whole_add (cuProlongate3D.cu:619-640): listed cells add their parent's value
template <typename T>
__global__ void __launch_bounds__(256) prolong_ix_kernel(T* __restrict__ v, const T* __restrict__ vc, Lvl<T> L,
                                                         int ncx, int ncy, const int4* __restrict__ seg, long nseg) {
    wp_pdl_enter();
    int x, y, z;
    if (!index_cell(seg, nseg, x, y, z)) return;
    v[y + (long)x * L.ny + (long)z * L.nx * L.ny] += vc[(y >> 1) + (long)(x >> 1) * ncy + (long)(z >> 1) * ncx * ncy];
}

// coarse face fractions: inject even faces along the face's own axis, average the (up to) two
// children along the two others (cuRestrict3D.cu:972-1145)
__global__ void coarsen_faces_kernel(float* __restrict__ dst, const float* __restrict__ src, int fnx, int fny, int fnz,
                                     int cnx, int cny, int cnz, int axis) {
    const int fe[3] = {fnx + (axis == 0), fny + (axis == 1), fnz + (axis == 2)};
    const int ce[3] = {cnx + (axis == 0), cny + (axis == 1), cnz + (axis == 2)};
    const long total = (long)ce[0] * ce[1] * ce[2];
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int c[3] = {(int)((t / ce[1]) % ce[0]), (int)(t % ce[1]), (int)(t / ((long)ce[0] * ce[1]))};
        int lo[3], cnt[3];
        for (int a = 0; a < 3; ++a) {
            if (a == axis) {
                int s = 2 * c[a];
                if ((fe[a] & 1) == 0 && c[a] == ce[a] - 1) s = 2 * c[a] - 1;
                lo[a] = s;
                cnt[a] = 1;
            } else {
                lo[a] = 2 * c[a];
                cnt[a] = (2 * c[a] + 1 < fe[a]) ? 2 : 1;
            }
        }
        float acc = 0.f;
        const float wt = 1.f / (float)(cnt[0] * cnt[1] * cnt[2]);
        for (int k = 0; k < cnt[2]; ++k)
            for (int i = 0; i < cnt[0]; ++i)
                for (int j = 0; j < cnt[1]; ++j)
                    acc += src[(lo[1] + j) + (long)(lo[0] + i) * fe[1] + (long)(lo[2] + k) * fe[0] * fe[1]];
        dst[c[1] + (long)c[0] * ce[1] + (long)c[2] * ce[0] * ce[1]] = acc * wt;
    }
}

struct Level {
    int n[3];
    long cells;
    float* frac[3];   // ax, ay, az (level-owned copies)
    float* fyc;       // ay re-laid per cell (lower y face), so y-quads of cells load with 128-bit accesses
    unsigned char* uni; // per (x, z) row: all of the row's interior face fractions are exactly 1
    unsigned char* tuni; // per (plane, tile) of the fused cycle kernels (tile_uni_kernel); levels whose
                         // extents fit those kernels (fz_level_ok) only
    int fz_fast;      // every cell's diagonal is positive on a fully open plane with the interior z
                      // factors: the fused kernels may take their straight-line path
    float* ccf;       // levels of at most kCoarseCells cells: per-cell stencils of the FP32 coarse cycle
    long long uni_rows; // rows flagged in uni
    double* tab64;    // per axis: glo[n], ghi[n], d[n]
    float* tab32;     // per axis: glo[n], ghi[n]
    float *v, *t, *f; // FP32 work
    double *v64, *t64, *f64;
    int zc[3];        // z planes per CTA of the column kernels (jacobi, coarse planes of resid_restrict,
                      // defect64); 0 = heuristic, set by wp_mgfrac3d_autotune
    float zc_ms[3];   // the autotuner's median time of the chosen chunk (0 = not tuned)
    int var[3];       // kernel variant per kind (jacobi: 0 = default registers, 1/2 = >= 3/4 CTAs per SM,
                      // 3 = two sweeps per launch, 4 = TMA-staged rows, 5 = cp.async-pipelined planes,
                      // 6 = one cell per thread; restrict: 0-2 register budgets, 3 = pipelined,
                      // 4 = one cell per thread; defect: 0 quads, 1 pipelined)
    int* err;         // the handle's device error flag (bounded waits of the TMA-staged kernel)
    // index-sparse cycle (built by the first wp_mgfrac3d_solve_index)
    unsigned* imask;  // per 32-cell segment of a row: the selected cells
    int4* iseg;       // the listed segments {x, z, y0, mask}, in memory order
    long long iseg_n; // listed segments
    long long icells; // selected cells (the reference's index size)
};

enum { kZcJacobi = 0, kZcRestrict = 1, kZcDefect = 2 };

// DRAM bytes of the face fractions one column-kernel pass over the level reads: 12 per cell of the
// rows that are not uniform, and the row flags
double frac_bytes(const Level& L) {
    const double rows = (double)L.n[0] * L.n[2];
    return 12.0 * (rows - (double)L.uni_rows) * L.n[1] + rows;
}

template <typename T>
Lvl<T> view(const Level& L);
template <>
Lvl<float> view<float>(const Level& L) {
    Lvl<float> o;
    o.nx = L.n[0]; o.ny = L.n[1]; o.nz = L.n[2];
    o.ax = L.frac[0]; o.ay = L.frac[1]; o.az = L.frac[2]; o.fyc = L.fyc; o.uni = L.uni;
    long off64 = 0, off32 = 0;
    for (int a = 0; a < 3; ++a) {
        o.glo[a] = L.tab32 + off32;
        o.ghi[a] = L.tab32 + off32 + L.n[a];
        o.d[a] = L.tab64 + off64 + 2 * L.n[a];
        off32 += 2 * L.n[a];
        off64 += 3 * L.n[a];
    }
    o.rwz = L.tab32 + off32;
    return o;
}
template <>
Lvl<double> view<double>(const Level& L) {
    Lvl<double> o;
    o.nx = L.n[0]; o.ny = L.n[1]; o.nz = L.n[2];
    o.ax = L.frac[0]; o.ay = L.frac[1]; o.az = L.frac[2]; o.fyc = L.fyc; o.uni = L.uni;
    long off64 = 0;
    for (int a = 0; a < 3; ++a) {
        o.glo[a] = L.tab64 + off64;
        o.ghi[a] = L.tab64 + off64 + L.n[a];
        o.d[a] = L.tab64 + off64 + 2 * L.n[a];
        off64 += 3 * L.n[a];
    }
    o.rwz = nullptr;  // the FP64 restriction divides in FP64
    return o;
}

dim3 grid_of(int nx, int ny, int nz) { return dim3(wp_cdiv(ny, 32), wp_cdiv(nx, 8), nz); }

// z planes per CTA so the grid holds about eight waves of 5 resident 256-thread CTAs per SM (a
// single wave leaves a tail that idles most SMs for the last CTAs)
int zchunk(int nx, int ny, int nz) {
    const long cols = (long)wp_cdiv(ny, 32) * wp_cdiv(nx, 8);
    const long want = 40L * wp_sm_count();
    long nzc = (want + cols - 1) / cols;
    if (nzc < 1) nzc = 1;
    if (nzc > nz) nzc = nz;
    return (int)((nz + nzc - 1) / nzc);
}
dim3 grid_z(int nx, int ny, int nz, int zc) { return dim3(wp_cdiv(ny, 32), wp_cdiv(nx, 8), wp_cdiv(nz, zc)); }

// levels whose y extent is a multiple of 4 run the quad kernels (when every array they read or
// write with 128-bit accesses is 16-byte aligned: caller-owned arrays may be offset views)
bool quad_ok(const Level& L) { return L.n[1] % 4 == 0; }
bool al16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// quad kernels: CTAs of 256 quads; about four waves of 4 resident CTAs per SM by default
int zchunk_q(int nx, int ny, int nz) {
    const long per_plane = wp_cdiv((size_t)nx * (ny / 4), 256);
    const long want = 16L * wp_sm_count();
    long nzc = (want + per_plane - 1) / per_plane;
    if (nzc < 1) nzc = 1;
    if (nzc > nz) nzc = nz;
    return (int)((nz + nzc - 1) / nzc);
}

int level_zc(const Level& L, int kind) {
    if (L.zc[kind] > 0) return L.zc[kind];
    const int zc = quad_ok(L) ? zchunk_q(L.n[0], L.n[1], L.n[2]) : zchunk(L.n[0], L.n[1], L.n[2]);
    return kind == kZcRestrict ? (zc + 1) / 2 : zc;
}

bool jacobi2_ok(const Level& L, const void* f) { return quad_ok(L) && al16(f) && L.n[2] >= 2; }

// the TMA-staged sweep: 3D levels with y rows of 16-byte multiples, aligned arrays
bool jacobi_ts_ok(const Level& L, const void* dst, const void* src, const void* f) {
    return quad_ok(L) && L.n[2] >= 2 && L.err && al16(dst) && al16(src) && al16(f) &&
           ts_smem_bytes(1, L.n[1]) <= 110 * 1024;
}

void launch_jacobi_ts(const Level& L, float* dst, const float* src, const float* f, float w, cudaStream_t s) {
    const int R = ts_rows(L.n[0], L.n[1]);
    const size_t smem = ts_smem_bytes(R, L.n[1]);
    if (wp_set_smem(jacobi_ts_kernel, smem) != cudaSuccess) return;
    const long W = (long)((L.n[0] + R - 1) / R) * L.n[2];
    const int grid = (int)std::min<long>(W, 2L * wp_sm_count());
    jacobi_ts_kernel<<<grid, TS_THREADS, smem, s>>>(dst, src, f, view<float>(L), w, R, L.err);
}

// one weighted-Jacobi sweep dst <- J(src) of level L
template <typename T>
void launch_jacobi(const Level& L, T* dst, const T* src, const T* f, T w, int zc, cudaStream_t s) {
    const Lvl<T> V = view<T>(L);
    const int var6 = sizeof(T) == 4 ? L.var[kZcJacobi] : 0;
    if (quad_ok(L) && al16(dst) && al16(src) && al16(f) && var6 != 6) {
        const dim3 g(wp_cdiv((size_t)L.n[0] * (L.n[1] / 4), 256), wp_cdiv(L.n[2], zc));
        const int var = var6;
        if (var == 4 && jacobi_ts_ok(L, dst, src, f)) {
            launch_jacobi_ts(L, (float*)dst, (const float*)src, (const float*)f, (float)w, s);
            return;
        }
        if constexpr (sizeof(T) == 4) {
            if (var == 5) {
                wp_launch_pdl(jacobi_qp_kernel<false>, g, 256, jp_smem_bytes(false), s, dst, src, f, V, w, zc, nullptr);
                return;
            }
        }
        if (var == 1) wp_launch_pdl(jacobi_q_mb_kernel<T, 3>, g, 256, 0, s, dst, src, f, V, w, zc, nullptr);
        else if (var == 2) wp_launch_pdl(jacobi_q_mb_kernel<T, 4>, g, 256, 0, s, dst, src, f, V, w, zc, nullptr);
        else wp_launch_pdl(jacobi_q_kernel<T>, g, 256, 0, s, dst, src, f, V, w, zc, nullptr);
    } else {
        jacobi_z_kernel<T, false><<<grid_z(L.n[0], L.n[1], L.n[2], zc), dim3(32, 8), 0, s>>>(dst, src, f, V, w, nullptr,
                                                                                          0, 0, zc);
    }
}


// One FP32 sweep of src whose result is added to p64 instead of stored (the level's tuned one-sweep
// quad kernel); false when the level's kernel has no such form (the caller then stores and adds).
bool jacobi_acc_ok(const Level& L, const void* src, const void* f, const double* p64) {
    return quad_ok(L) && al16(src) && al16(f) && al16(p64) && (L.var[kZcJacobi] <= 2 || L.var[kZcJacobi] == 5);
}
void launch_jacobi_acc(const Level& L, const float* src, const float* f, float w, int zc, double* p64,
                       cudaStream_t s) {
    const int var = L.var[kZcJacobi];
    const Lvl<float> V = view<float>(L);
    const dim3 g(wp_cdiv((size_t)L.n[0] * (L.n[1] / 4), 256), wp_cdiv(L.n[2], zc));
    if (var == 1) wp_launch_pdl(jacobi_q_mb_kernel<float, 3, true>, g, 256, 0, s, nullptr, src, f, V, w, zc, p64);
    else if (var == 5) {
        wp_set_smem(jacobi_qp_kernel<true>, jp_smem_bytes(true));
        wp_launch_pdl(jacobi_qp_kernel<true>, g, 256, jp_smem_bytes(true), s, nullptr, src, f, V, w, zc, p64);
    }
    else if (var == 2)
        wp_launch_pdl(jacobi_q_mb_kernel<float, 4, true>, g, 256, 0, s, nullptr, src, f, V, w, zc, p64);
    else wp_launch_pdl(jacobi_q_kernel<float, true>, g, 256, 0, s, nullptr, src, f, V, w, zc, p64);
}

// two sweeps dst <- J(J(src)) in one pass (jacobi2_q_kernel)
template <typename T>
void launch_jacobi2(const Level& L, T* dst, const T* src, const T* f, T w, int zc, cudaStream_t s) {
    const int nty = (L.n[1] / 4 + J2_Q - 1) / J2_Q, ntx = (L.n[0] + J2_R - 1) / J2_R;
    jacobi2_q_kernel<T><<<dim3(ntx * nty, wp_cdiv(L.n[2], zc)), J2_THREADS, 0, s>>>(dst, src, f, view<T>(L), w, zc,
                                                                                   nty);
}

// coarse f of C = restriction of the residual f - A v of level L (czc coarse planes per CTA)
template <typename T>
void launch_resid_restrict(const Level& L, const Level& C, T* fc, const T* v, const T* f, int czc, cudaStream_t s) {
    const Lvl<T> V = view<T>(L);
    if (quad_ok(L) && C.n[1] * 2 == L.n[1] && al16(v) && al16(f) && (sizeof(T) != 4 || L.var[kZcRestrict] != 4)) {
        const dim3 g(wp_cdiv((size_t)C.n[0] * (L.n[1] / 4) * 2, 256), wp_cdiv(C.n[2], czc));
        const int var = sizeof(T) == 4 ? L.var[kZcRestrict] : 0;
        if constexpr (sizeof(T) == 4) {
            if (var == 3) {
                wp_launch_pdl(resid_restrict_qp_kernel, g, 256, jp_smem_bytes(false), s, fc, v, f, V, C.n[0], C.n[1],
                              C.n[2], czc);
                return;
            }
        }
        if (var == 1) wp_launch_pdl(resid_restrict_q_kernel<T, 3>, g, 256, 0, s, fc, v, f, V, C.n[0], C.n[1], C.n[2], czc);
        else if (var == 2)
            wp_launch_pdl(resid_restrict_q_kernel<T, 4>, g, 256, 0, s, fc, v, f, V, C.n[0], C.n[1], C.n[2], czc);
        else wp_launch_pdl(resid_restrict_q_kernel<T>, g, 256, 0, s, fc, v, f, V, C.n[0], C.n[1], C.n[2], czc);
    } else {
        const dim3 g(wp_cdiv(L.n[1], 32), wp_cdiv(L.n[0], 8), wp_cdiv(C.n[2], czc));
        resid_restrict_z_kernel<T><<<g, dim3(32, 8), 0, s>>>(fc, v, f, V, C.n[0], C.n[1], C.n[2], czc);
    }
}

// FP64 defect of the finest level into acc[0] (see defect64_z_kernel)
template <typename TP>
void launch_defect64(const Level& L, float* r32, const TP* p, const float* f, double m, const double* msum,
                     double* acc, int zc, cudaStream_t s) {
    const Lvl<double> V = view<double>(L);
    if (quad_ok(L) && al16(r32) && al16(p) && al16(f)) {
        const dim3 g(wp_cdiv((size_t)L.n[0] * (L.n[1] / 4), 256), wp_cdiv(L.n[2], zc));
        if constexpr (sizeof(TP) == 8) {
            if (L.var[kZcDefect] == 1) {
                wp_set_smem(defect64_qp_kernel, jp_smem_bytes(true) - (size_t)JP_DEPTH * 256 * 16);
                wp_launch_pdl(defect64_qp_kernel, g, 256, jp_smem_bytes(true) - (size_t)JP_DEPTH * 256 * 16, s, r32,
                              (const double*)p, f, V, m, msum, acc, zc);
                return;
            }
        }
        wp_launch_pdl(defect64_q_kernel<TP>, g, 256, 0, s, r32, p, f, V, m, msum, acc, zc);
    } else {
        defect64_z_kernel<TP><<<grid_z(L.n[0], L.n[1], L.n[2], zc), dim3(32, 8), 0, s>>>(r32, p, f, V, m, msum, acc,
                                                                                       zc);
    }
}

template <typename T>
void launch_prolong_tri(const Level& L, const Level& C, T* v, const T* vc, cudaStream_t s) {
    if (quad_ok(L) && al16(v)) {
        const dim3 g(wp_cdiv((size_t)L.n[0] * (L.n[1] / 4), 256), L.n[2]);
        wp_launch_pdl(prolong_tri_q_kernel<T>, g, 256, 0, s, v, vc, L.n[0], L.n[1], L.n[2], C.n[0], C.n[1], C.n[2]);
    } else {
        prolong_tri_add_kernel<T><<<grid_of(L.n[0], L.n[1], L.n[2]), dim3(32, 8), 0, s>>>(v, vc, L.n[0], L.n[1], L.n[2],
                                                                                         C.n[0], C.n[1], C.n[2]);
    }
}

// levels the fused cycle kernels handle: whole 32 x 32 (x, y) tiles and an even number of planes
bool fz_level_ok(const int* n) { return n[0] % fz::TX == 0 && n[1] % fz::TY == 0 && n[2] >= 2 && n[2] % 2 == 0; }

// z planes per CTA (even): `want`, or 16.  Chunks of 16 planes (one warm-up pair of planes per
// eight) keep several waves of CTAs, so the hardware scheduler evens out tiles that cross solids
// (their planes take the slower general path); at 256^3 with four spheres 16 beat 8, 24-128 and a
// single wave of one chunk per resident slot.
int fz_zchunk(const Level& L, int want) {
    int zc = want > 0 ? want : 16;
    zc += zc & 1;
    // a chunk's planes and their pipeline halo fit the kernels' plane table
    return std::min(std::min(zc, L.n[2] + (L.n[2] & 1)), fz::ZT - 6);
}

// pre-smoothing + residual restriction of level L into fc (cycle_down_kernel); v0 NULL: from zero.
// False when a tensor map cannot be made.
bool launch_cycle_down(const Level& L, float* dst, float* fc, const float* v0, const float* f, float w, int zc,
                       cudaStream_t s) {
    CUtensorMap mv, mf;
    if (!wptc::map_f32_3d(&mf, f, L.n[1], L.n[0], L.n[2], fz::RY, fz::RX)) return false;
    if (v0 && !wptc::map_f32_3d(&mv, v0, L.n[1], L.n[0], L.n[2], fz::RY, fz::RX + 2)) return false;
    if (!v0) mv = mf;  // not read
    const dim3 g((L.n[0] / fz::TX) * (L.n[1] / fz::TY), wp_cdiv(L.n[2], zc));
    const Lvl<float> V = view<float>(L);
    const unsigned char* tu = L.tuni;
    if (v0) {
        if (wp_set_smem(cycle_down_kernel<false>, fz::smem_bytes) != cudaSuccess) return false;
        wp_launch_pdl(cycle_down_kernel<false>, g, fz::THREADS, fz::smem_bytes, s, mv, mf, dst, fc, V, tu, w, zc,
                      L.fz_fast, L.err);
    } else {
        if (wp_set_smem(cycle_down_kernel<true>, fz::smem_bytes) != cudaSuccess) return false;
        wp_launch_pdl(cycle_down_kernel<true>, g, fz::THREADS, fz::smem_bytes, s, mv, mf, dst, fc, V, tu, w, zc,
                      L.fz_fast, L.err);
    }
    return true;
}

// prolongation of the coarse correction vc + post-smoothing of vin (cycle_up_kernel): into dst, or
// added to p64 when p64 is given
bool launch_cycle_up(const Level& L, const Level& C, float* dst, double* p64, const float* vin, const float* vc,
                     const float* f, float w, int zc, cudaStream_t s) {
    (void)C;
    CUtensorMap mv, mf;
    if (!wptc::map_f32_3d(&mf, f, L.n[1], L.n[0], L.n[2], fz::RY, fz::RX)) return false;
    if (!wptc::map_f32_3d(&mv, vin, L.n[1], L.n[0], L.n[2], fz::RY, fz::RX + 2)) return false;
    const dim3 g((L.n[0] / fz::TX) * (L.n[1] / fz::TY), wp_cdiv(L.n[2], zc));
    const Lvl<float> V = view<float>(L);
    const unsigned char* tu = L.tuni;
    if (p64) {
        if (wp_set_smem(cycle_up_kernel<true>, fz::smem_bytes) != cudaSuccess) return false;
        wp_launch_pdl(cycle_up_kernel<true>, g, fz::THREADS, fz::smem_bytes, s, mv, mf, (float*)nullptr, p64, vc, V, tu, w,
                      zc, L.fz_fast, L.err);
    } else {
        if (wp_set_smem(cycle_up_kernel<false>, fz::smem_bytes) != cudaSuccess) return false;
        wp_launch_pdl(cycle_up_kernel<false>, g, fz::THREADS, fz::smem_bytes, s, mv, mf, dst, (double*)nullptr, vc, V, tu,
                      w, zc, L.fz_fast, L.err);
    }
    return true;
}

}  // namespace

struct wp_mgfrac3d {
    int dims;          // 2 or 3 (2D problems use nz = 1)
    int last64;        // 0: none, 1: p64 (mixed), 2: lv[0].v64 (fp64) holds the last FP64 iterate
    int nl;
    Level lv[kMaxLevels];
    int coarsest_iters;
    double* acc;       // device reduction slots; then the int error flag (acc + 4) and the grid
                       // barrier words of mid_cycle_kernel (8 bytes further)
    int mid_on;        // run the levels below the finest as one persistent launch (autotuned, default on)
    int mid_forbid;    // never (handles whose cycles share the GPU with concurrent graph branches)
    int mid_grid;      // its CTAs (one per SM; 0 = not yet known, -1 = not possible on this device)
    double* p64;       // FP64 iterate for mixed precision
    float* r32;        // FP32 defect (right-hand side of correction cycles)
    const float* fin;  // finest right-hand side of the current solve
    const double* fin64;
    float* ccf_all;    // the coarse levels' stencils (Level::ccf points into it)
    int tune_gen;      // bumped by every change of a level's tile or kernel variant
    // device-side cycle loop of the mixed-precision tolerance solve (see solve_mixed_graph)
    cudaGraph_t loop_graph;
    cudaGraphExec_t loop_exec;
    void* loop_state;  // device MgLoop
    cudaStream_t loop_cap; // private stream the loop is captured on (capture needs a non-default stream)
    int loop_broken;   // capture or instantiation failed once: the host loop is used from then on
    const float* loop_f;
    int loop_key[7];   // nu1, nu2, prolongation, full-multigrid first cycle, tune_gen, device, inner cycles
    double loop_omega;
    long long loop_launches[2]; // kernels of the first cycle's graph part and of one loop body
    int fz_on;         // run the V(2,2) FP32 cycle of level 0 as the two fused kernels where it fits
    int fz_zc;         // their z planes per CTA (0 = heuristic)
    int ix_built;      // the index lists of every level exist
    float* ix_r;       // residual workspace of the index-sparse cycle, shared by the levels (finest size)
    double* ix_r64;    // the same for the FP64 cycle
};

namespace {

wp_status build_hierarchy(wp_mgfrac3d* h, const float* ax, const float* ay, const float* az, int nx, int ny, int nz,
                          double dx, double dy, double dz, cudaStream_t s) {
    int n[3] = {nx, ny, nz};
    const int dims = h->dims;
    auto mn = [&](const int* e) { return dims == 2 ? (e[0] < e[1] ? e[0] : e[1]) : std::min(e[0], std::min(e[1], e[2])); };
    std::vector<double> hd[3];
    hd[0].assign(nx, dx);
    hd[1].assign(ny, dy);
    hd[2].assign(nz, dz);
    int nl = 0;
    while (mn(n) > 1 && nl < kMaxLevels) {
        Level& L = h->lv[nl];
        for (int a = 0; a < 3; ++a) L.n[a] = n[a];
        L.cells = (long)n[0] * n[1] * n[2];
        const long fs[3] = {(long)(n[0] + 1) * n[1] * n[2], (long)n[0] * (n[1] + 1) * n[2],
                            dims == 2 ? 1 : (long)n[0] * n[1] * (n[2] + 1)};
        for (int a = 0; a < 3; ++a) WP_CUDA_TRY(cudaMalloc((void**)&L.frac[a], sizeof(float) * fs[a]));
        if (nl == 0) {
            WP_CUDA_TRY(cudaMemcpyAsync(L.frac[0], ax, sizeof(float) * fs[0], cudaMemcpyDeviceToDevice, s));
            WP_CUDA_TRY(cudaMemcpyAsync(L.frac[1], ay, sizeof(float) * fs[1], cudaMemcpyDeviceToDevice, s));
            if (dims == 3) WP_CUDA_TRY(cudaMemcpyAsync(L.frac[2], az, sizeof(float) * fs[2], cudaMemcpyDeviceToDevice, s));
            else WP_CUDA_TRY(cudaMemsetAsync(L.frac[2], 0, sizeof(float), s));
        } else {
            const Level& F = h->lv[nl - 1];
            for (int a = 0; a < dims; ++a) {
                WP_KERNEL("coarsen_faces", 4.0 * 9 * fs[a], s,
                          coarsen_faces_kernel<<<wp_cdiv(fs[a], 256) > 4096 ? 4096 : wp_cdiv(fs[a], 256), 256, 0, s>>>(
                              L.frac[a], F.frac[a], F.n[0], F.n[1], F.n[2], n[0], n[1], n[2], a));
            }
            if (dims == 2) WP_CUDA_TRY(cudaMemsetAsync(L.frac[2], 0, sizeof(float), s));
        }
        WP_CUDA_TRY(cudaMalloc((void**)&L.fyc, sizeof(float) * L.cells));
        WP_KERNEL("fyc", 8.0 * L.cells, s,
                  fyc_kernel<<<std::min<unsigned>(wp_cdiv(L.cells, 256), 4096), 256, 0, s>>>(L.fyc, L.frac[1], n[0],
                                                                                             n[1], L.cells));
        WP_CUDA_TRY(cudaMalloc((void**)&L.uni, (size_t)n[0] * n[2]));
        WP_KERNEL("uniform_rows", 16.0 * L.cells, s,
                  uniform_rows_kernel<<<std::min<unsigned>(wp_cdiv((long)n[0] * n[2] * 32, 256), 4096), 256, 0, s>>>(
                      L.uni, L.frac[0], L.fyc, L.frac[2], n[0], n[1], n[2]));
        {
            std::vector<unsigned char> u((size_t)n[0] * n[2]);
            WP_CUDA_TRY(cudaMemcpyAsync(u.data(), L.uni, u.size(), cudaMemcpyDeviceToHost, s));
            WP_CUDA_TRY(cudaStreamSynchronize(s));
            L.uni_rows = 0;
            for (unsigned char b : u) L.uni_rows += b != 0;
        }
        if (dims == 3 && fz_level_ok(n)) {
            const int ntiles = (n[0] / fz::TX) * (n[1] / fz::TY);
            WP_CUDA_TRY(cudaMalloc((void**)&L.tuni, (size_t)ntiles * n[2]));
            Lvl<float> V{};
            V.nx = n[0]; V.ny = n[1]; V.nz = n[2];
            V.ax = L.frac[0]; V.ay = L.frac[1]; V.az = L.frac[2]; V.fyc = L.fyc;
            WP_KERNEL("tile_uniform", 12.0 * L.cells, s,
                      tile_uni_kernel<<<dim3(ntiles, n[2]), 256, 0, s>>>(L.tuni, V));
            if (nl == 0) {
                // the fused kernels' shared-memory limits, set here rather than while a cycle is captured
                WP_CUDA_TRY(wp_set_smem(cycle_down_kernel<true>, fz::smem_bytes));
                WP_CUDA_TRY(wp_set_smem(cycle_down_kernel<false>, fz::smem_bytes));
                WP_CUDA_TRY(wp_set_smem(cycle_up_kernel<true>, fz::smem_bytes));
                WP_CUDA_TRY(wp_set_smem(cycle_up_kernel<false>, fz::smem_bytes));
            }
        }
        // spacing tables; 2D problems have a single z layer with no z faces (tables all zero)
        std::vector<double> t64;
        std::vector<float> t32;
        for (int a = 0; a < 3; ++a) {
            const int m = n[a];
            std::vector<double> lo(m, 0.0), hi(m, 0.0);
            for (int i = 0; i < m; ++i) {
                if (i > 0) lo[i] = 2.0 / ((hd[a][i - 1] + hd[a][i]) * hd[a][i]);
                if (i < m - 1) hi[i] = 2.0 / ((hd[a][i + 1] + hd[a][i]) * hd[a][i]);
            }
            t64.insert(t64.end(), lo.begin(), lo.end());
            t64.insert(t64.end(), hi.begin(), hi.end());
            t64.insert(t64.end(), hd[a].begin(), hd[a].end());
            for (double v : lo) t32.push_back((float)v);
            for (double v : hi) t32.push_back((float)v);
        }
        // after the three axes' factors: the z restriction weights (the FP64 quotient the restriction
        // forms per fine plane, rounded once; the kernels read it instead of dividing)
        for (int z = 0; z < n[2]; ++z) {
            const int zb = z & ~1;
            const double sz = hd[2][zb] + (zb + 1 < n[2] ? hd[2][zb + 1] : 0.0);
            t32.push_back((float)(hd[2][z] / sz));
        }
        {
            // smallest diagonal of a fully open cell (the fused kernels' straight-line path divides by
            // none): the least lower + upper factor per axis, z at the interior reference plane
            float mn[2] = {0.f, 0.f};
            for (int a = 0; a < 2; ++a) {
                const float* lo = t32.data() + 2 * (size_t)(a == 0 ? 0 : n[0]);
                const float* hi = lo + n[a];
                mn[a] = lo[0] + hi[0];
                for (int i = 1; i < n[a]; ++i) mn[a] = std::min(mn[a], lo[i] + hi[i]);
            }
            const float* zlo = t32.data() + 2 * (size_t)(n[0] + n[1]);
            const int zr = n[2] / 2;
            const float dmin = ((mn[1] + mn[0]) + zlo[zr]) + zlo[n[2] + zr];
            L.fz_fast = dmin > 1e-10f ? 1 : 0;
        }
        WP_CUDA_TRY(cudaMalloc((void**)&L.tab64, sizeof(double) * t64.size()));
        WP_CUDA_TRY(cudaMalloc((void**)&L.tab32, sizeof(float) * t32.size()));
        WP_CUDA_TRY(cudaMemcpy(L.tab64, t64.data(), sizeof(double) * t64.size(), cudaMemcpyHostToDevice));
        WP_CUDA_TRY(cudaMemcpy(L.tab32, t32.data(), sizeof(float) * t32.size(), cudaMemcpyHostToDevice));
        WP_CUDA_TRY(cudaMalloc((void**)&L.v, sizeof(float) * L.cells));
        WP_CUDA_TRY(cudaMalloc((void**)&L.t, sizeof(float) * L.cells));
        WP_CUDA_TRY(cudaMalloc((void**)&L.f, sizeof(float) * L.cells));
        WP_CUDA_TRY(cudaMemsetAsync(L.v, 0, sizeof(float) * L.cells, s));
        ++nl;
        // next level: ceil halving, coarse spacing = sum of the two fine spacings (cuRestrictDx)
        for (int a = 0; a < dims; ++a) {
            const int m = wp_half_up(n[a]);
            std::vector<double> c(m);
            for (int i = 0; i < m; ++i) c[i] = hd[a][2 * i] + (2 * i + 1 < n[a] ? hd[a][2 * i + 1] : 0.0);
            hd[a] = c;
            n[a] = m;
        }
    }
    h->nl = nl;
    // per-cell stencils of the levels of at most kCoarseCells cells (a suffix of the hierarchy), in
    // one block in level order so that any coarse-cycle pack finds its stencils contiguous
    long cf = 0;
    for (int l = 0; l < nl; ++l)
        if (h->lv[l].cells <= kCoarseCells) cf += (long)kCcf * h->lv[l].cells;
    if (cf > 0) {
        WP_CUDA_TRY(cudaMalloc((void**)&h->ccf_all, sizeof(float) * cf));
        long off = 0;
        for (int l = 0; l < nl; ++l) {
            Level& L = h->lv[l];
            if (L.cells > kCoarseCells) continue;
            L.ccf = h->ccf_all + off;
            off += (long)kCcf * L.cells;
            WP_KERNEL("cc_coeff", 40.0 * L.cells, s,
                      cc_coeff_kernel<<<wp_cdiv(L.cells, 256), 256, 0, s>>>(L.ccf, view<float>(L)));
        }
    }
    return WP_OK;
}

wp_status ensure_fp64(wp_mgfrac3d* h) {
    for (int l = 0; l < h->nl; ++l) {
        Level& L = h->lv[l];
        if (L.v64) continue;
        WP_CUDA_TRY(cudaMalloc((void**)&L.v64, sizeof(double) * L.cells));
        WP_CUDA_TRY(cudaMalloc((void**)&L.t64, sizeof(double) * L.cells));
        WP_CUDA_TRY(cudaMalloc((void**)&L.f64, sizeof(double) * L.cells));
    }
    return WP_OK;
}

template <typename T>
struct Bufs;
template <>
struct Bufs<float> {
    static float*& v(Level& L) { return L.v; }
    static float*& t(Level& L) { return L.t; }
    static float*& f(Level& L) { return L.f; }
};
template <>
struct Bufs<double> {
    static double*& v(Level& L) { return L.v64; }
    static double*& t(Level& L) { return L.t64; }
    static double*& f(Level& L) { return L.f64; }
};

// profile names: the finest level is reported apart (it carries the roofline of the cycle)
// acc64 (FP32 levels): the last sweep adds its result to acc64 instead of storing it, when the
// level's kernel allows (*added reports it; the level's v then holds no meaningful values)
template <typename T>
wp_status smooth(Level& L, const T* f, int sweeps, T w, cudaStream_t s, bool finest = false, double* acc64 = nullptr,
                 bool* added = nullptr) {
    const int zc = level_zc(L, kZcJacobi);
    // the variant is tuned on the FP32 kernels; FP64 smoothing keeps one sweep per launch
    const bool fused = sizeof(T) == 4 && L.var[kZcJacobi] == 3 && jacobi2_ok(L, f);
    for (int k = 0; k < sweeps;) {
        if (sizeof(T) == 4 && acc64 && k == sweeps - 1 && jacobi_acc_ok(L, Bufs<T>::v(L), f, acc64)) {
            WP_KERNEL(finest ? "jacobi_finest_update" : "jacobi_update",
                      (double)L.cells * (2.0 * sizeof(T) + 16.0) + frac_bytes(L), s,
                      launch_jacobi_acc(L, (const float*)Bufs<T>::v(L), (const float*)f, (float)w, zc, acc64, s));
            *added = true;
            T* tmp = Bufs<T>::v(L);
            Bufs<T>::v(L) = Bufs<T>::t(L);
            Bufs<T>::t(L) = tmp;
            break;
        }
        if (fused && sweeps - k >= 2) {
            // two sweeps, one pass: algorithmic bytes are those of one sweep
            WP_KERNEL(finest ? "jacobi2_finest" : "jacobi2", (double)L.cells * (3.0 * sizeof(T) + 12.0), s,
                      launch_jacobi2<T>(L, Bufs<T>::t(L), Bufs<T>::v(L), f, w, zc, s));
            k += 2;
        } else {
            WP_KERNEL(finest ? "jacobi_finest" : "jacobi", (double)L.cells * 3.0 * sizeof(T) + frac_bytes(L), s,
                      launch_jacobi<T>(L, Bufs<T>::t(L), Bufs<T>::v(L), f, w, zc, s));
            k += 1;
        }
        T* tmp = Bufs<T>::v(L);
        Bufs<T>::v(L) = Bufs<T>::t(L);
        Bufs<T>::t(L) = tmp;
    }
    return WP_OK;
}

// The V-cycle below the finest level (from level l1, v = 0) as one mid_cycle_kernel launch when the
// levels allow it (FP32, trilinear prolongation, nu1 >= 1, quad levels down to a lean coarse pack);
// sets *done.  The host mirrors every ping-pong swap the phases perform.
wp_status mid_cycle(wp_mgfrac3d* h, int l1, int nu1, int nu2, float w, int prolong, cudaStream_t s, bool* done) {
    *done = false;
    if (!h->mid_on || h->mid_forbid || h->dims != 3 || h->mid_grid < 0 || prolong != WP_PROLONG_TRILINEAR ||
        nu1 < 1 || l1 < 1)
        return WP_OK;
    // the coarse pack starts at the first level the fused coarse cycle takes
    int lc = -1;
    for (int l = l1; l < h->nl - 1 && lc < 0; ++l) {
        long pack = 0;
        for (int k = l; k < h->nl; ++k) pack += h->lv[k].cells;
        if (h->lv[l].cells <= kCoarseCells && h->nl - l <= kCoarseMax && pack <= kCoarseSmemCells) lc = l;
    }
    if (lc <= l1 || lc - l1 + 1 > kMidLevels) return WP_OK;
    for (int l = l1; l < lc; ++l) {
        Level& L = h->lv[l];
        const Level& C = h->lv[l + 1];
        if (!quad_ok(L) || C.n[1] * 2 != L.n[1] || !al16(L.v) || !al16(L.t) || !al16(L.f)) return WP_OK;
    }
    LPack Q;
    Q.n = h->nl - lc;
    for (int k = 0; k < Q.n; ++k) {
        Level& E = h->lv[lc + k];
        if (!E.ccf) return WP_OK;
        Q.lv[k] = {E.n[0], E.n[1], E.n[2], E.ccf, E.v, E.t, E.f};
    }
    const size_t lean_bytes = sizeof(float) * (size_t)lean_smem_floats(Q);
    if (lean_bytes > kLeanSmemMax) return WP_OK;
    if (h->mid_grid == 0) {
        int per_sm = 0;
        if (wp_set_smem(mid_cycle_kernel, kLeanSmemMax) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mid_cycle_kernel, 1024, kLeanSmemMax) !=
                cudaSuccess ||
            per_sm < 1) {
            (void)cudaGetLastError();
            h->mid_grid = -1;
            return WP_OK;
        }
        h->mid_grid = wp_sm_count();
    }
    MidPack P;
    memset(&P, 0, sizeof(P));
    for (int l = l1; l <= lc; ++l) P.L[l - l1] = view<float>(h->lv[l]);
    auto add = [&](int type, int l, float* dst, const float* src, const float* f, int zc, int gx, int gy) {
        MidPhase& q = P.ph[P.nph++];
        q.type = type;
        q.level = l - l1;
        q.dst = dst;
        q.src = src;
        q.f = f;
        q.zc = zc;
        q.gx = gx;
        q.gy = gy;
    };
    const int phases = (lc - l1) * (nu1 + 1 + 1 + nu2) + 1;
    if (phases > kMidPhases) return WP_OK;
    auto quads = [](const Level& L) { return (int)wp_cdiv((size_t)L.n[0] * (L.n[1] / 4), 256); };
    for (int l = l1; l < lc; ++l) {
        Level& L = h->lv[l];
        Level& C = h->lv[l + 1];
        const int zc = 1;  // as many work units as possible: the phases are short
        add(MP_SWEEP0, l, L.t, nullptr, L.f, zc, quads(L), (int)wp_cdiv(L.n[2], zc));
        std::swap(L.v, L.t);
        for (int k = 1; k < nu1; ++k) {
            add(MP_SWEEP, l, L.t, L.v, L.f, zc, quads(L), (int)wp_cdiv(L.n[2], zc));
            std::swap(L.v, L.t);
        }
        const int czc = 1;
        add(MP_RESTRICT, l, C.f, L.v, L.f, czc, (int)wp_cdiv((size_t)C.n[0] * (L.n[1] / 4) * 2, 256),
            (int)wp_cdiv(C.n[2], czc));
    }
    add(MP_COARSE, lc, nullptr, nullptr, nullptr, 0, 0, 0);
    for (int k = 0; k < Q.n; ++k) {
        Level& E = h->lv[lc + k];
        const int swaps = (k == Q.n - 1) ? h->coarsest_iters : nu1 + nu2;
        if (swaps & 1) std::swap(E.v, E.t);
    }
    for (int l = lc - 1; l >= l1; --l) {
        Level& L = h->lv[l];
        Level& C = h->lv[l + 1];
        const int zc = 1;
        add(MP_PROLONG, l, L.v, C.v, nullptr, 0, quads(L), L.n[2]);
        for (int k = 0; k < nu2; ++k) {
            add(MP_SWEEP, l, L.t, L.v, L.f, zc, quads(L), (int)wp_cdiv(L.n[2], zc));
            std::swap(L.v, L.t);
        }
    }
    P.coarse = Q;
    P.nu1 = nu1;
    P.nu2 = nu2;
    P.citers = h->coarsest_iters;
    P.prolong = prolong;
    P.w = w;
    P.err = reinterpret_cast<int*>(h->acc + 4);
    P.bar = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(h->acc + 4) + 8);
    int wh_at = 0;
    P.lim = wptc::kWaitLimitNs;
    P.withhold = wp_take_withhold(WP_WAIT_SITE_GRID_BARRIER, s, &wh_at, &P.lim) ? 1 : 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(h->mid_grid);
    cfg.blockDim = dim3(1024);
    cfg.dynamicSmemBytes = lean_bytes;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    double bytes = 0.0;
    for (int l = l1; l < lc; ++l)
        bytes += (double)h->lv[l].cells * 4.0 * (3.0 * (nu1 + nu2) + 8.0) + 2.0 * frac_bytes(h->lv[l]) * (nu1 + nu2 + 1);
    // a barrier that gave up in an earlier launch may have left arrivals counted
    WP_CUDA_TRY(cudaMemsetAsync(P.bar, 0, sizeof(unsigned), s));
    WP_KERNEL("mid_cycle", bytes, s, cudaLaunchKernelEx(&cfg, mid_cycle_kernel, P));
    *done = true;
    return WP_OK;
}

// The coarsest solve (cuWjFrac3D_kernel_n, cuWeightedJacobi3D.cu:1473-1545) from the level's v:
// in one CTA when the level fits its shared memory, else as ordinary sweeps.
template <typename T>
wp_status coarsest_solve(wp_mgfrac3d* h, Level& L, const T* f, T w, cudaStream_t s) {
    const size_t smem = 2 * sizeof(T) * L.cells;
    if (smem <= 200 * 1024) {
        auto k = coarsest_kernel<T>;
        WP_CUDA_TRY(wp_set_smem(k, smem));
        const int nt = (int)std::min<long>(1024, (L.cells + 31) / 32 * 32);
        WP_KERNEL("coarsest", (double)L.cells * (3.0 * sizeof(T) + 12.0), s,
                  k<<<1, nt, smem, s>>>(Bufs<T>::v(L), f, view<T>(L), w, h->coarsest_iters));
        return WP_OK;
    }
    return smooth<T>(L, f, h->coarsest_iters, w, s);
}

// One V-cycle at level l from the level's current v, or (clear_v) from v = 0: then v is neither
// cleared nor read -- the first sweep is jacobi0_q_kernel where the level's kernel allows, otherwise
// v is cleared first -- and below kCoarseCells the single-launch coarse cycle takes over.
// acc64 / added: see smooth (the finest level's last post-sweep adds into acc64 when it can).
template <typename T>
wp_status vcycle(wp_mgfrac3d* h, int l, const T* f, int nu1, int nu2, T w, int prolong, cudaStream_t s, bool clear_v,
                 double* acc64 = nullptr, bool* added = nullptr) {
    Level& L = h->lv[l];
    const dim3 g = grid_of(L.n[0], L.n[1], L.n[2]);
    wp_status st;
    if constexpr (sizeof(T) == 4) {
        if (clear_v && l >= 1) {
            bool done = false;
            if ((st = mid_cycle(h, l, nu1, nu2, (float)w, prolong, s, &done)) != WP_OK) return st;
            if (done) return WP_OK;
        }
    }
    long pack_cells = 0;
    for (int k = l; k < h->nl; ++k) pack_cells += h->lv[k].cells;
    if (clear_v && l > 0 && l < h->nl - 1 && L.cells <= kCoarseCells && h->nl - l <= kCoarseMax &&
        f == Bufs<T>::f(L) && pack_cells <= kCoarseSmemCells) {
        // the rest of the cycle in one launch; the host mirrors the buffer swaps it performs
        bool lean = sizeof(T) == 4;
        LPack Q;
        Q.n = h->nl - l;
        for (int k = 0; k < Q.n && lean; ++k) {
            Level& E = h->lv[l + k];
            lean = E.ccf != nullptr;
            Q.lv[k] = {E.n[0], E.n[1], E.n[2], E.ccf, (float*)Bufs<T>::v(E), (float*)Bufs<T>::t(E),
                       (const float*)Bufs<T>::f(E)};
        }
        const size_t lean_bytes = lean ? sizeof(float) * (size_t)lean_smem_floats(Q) : 0;
        if (lean && lean_bytes <= kLeanSmemMax) {
            WP_CUDA_TRY(wp_set_smem(coarse_cycle_lean_kernel, kLeanSmemMax));
            WP_KERNEL("coarse_cycle", (double)L.cells * (3.0 * sizeof(T) + 12.0) * (nu1 + nu2 + 2), s,
                      wp_launch_pdl(coarse_cycle_lean_kernel, 1, 1024, lean_bytes, s, Q, nu1, nu2, (float)w,
                                    h->coarsest_iters, prolong));
            for (int k = 0; k < Q.n; ++k) {
                Level& E = h->lv[l + k];
                const int swaps = (k == Q.n - 1) ? h->coarsest_iters : nu1 + nu2;
                if (swaps & 1) std::swap(Bufs<T>::v(E), Bufs<T>::t(E));
            }
            return WP_OK;
        }
        const size_t smem_max = 3 * sizeof(T) * (size_t)kCoarseSmemCells;
        WP_CUDA_TRY(wp_set_smem(coarse_cycle_kernel<T>, smem_max));
        CPack<T> P;
        P.n = h->nl - l;
        for (int k = 0; k < P.n; ++k) {
            Level& Q = h->lv[l + k];
            P.lv[k].L = view<T>(Q);
            P.lv[k].v = Bufs<T>::v(Q);
            P.lv[k].t = Bufs<T>::t(Q);
            P.lv[k].f = Bufs<T>::f(Q);
        }
        WP_KERNEL("coarse_cycle", (double)L.cells * (3.0 * sizeof(T) + 12.0) * (nu1 + nu2 + 2), s,
                  coarse_cycle_kernel<T><<<1, 1024, 3 * sizeof(T) * pack_cells, s>>>(P, nu1, nu2, w,
                                                                                      h->coarsest_iters, prolong));
        for (int k = 0; k < P.n; ++k) {
            Level& Q = h->lv[l + k];
            const int swaps = (k == P.n - 1) ? h->coarsest_iters : nu1 + nu2;
            if (swaps & 1) std::swap(Bufs<T>::v(Q), Bufs<T>::t(Q));
        }
        return WP_OK;
    }
    if (l < h->nl - 1) {
        if constexpr (sizeof(T) == 4) {
            // level 0's V(2,2) cycle as two fused passes (wp_mg_fused.cuh): pre-smoothing + residual
            // restriction, then prolongation + post-smoothing (+ the refinement update)
            Level& C = h->lv[l + 1];
            if (l == 0 && h->fz_on && L.tuni && h->dims == 3 && prolong == WP_PROLONG_TRILINEAR && nu1 == 2 &&
                nu2 == 2 && C.n[0] * 2 == L.n[0] && C.n[1] * 2 == L.n[1] && C.n[2] * 2 == L.n[2] && al16(f) &&
                al16(L.v) && al16(L.t) && wptc::encode_tiled()) {
                const int zc = fz_zchunk(L, h->fz_zc);
                const float* v0 = clear_v ? nullptr : L.v;
                bool okl = true;
                WP_KERNEL(v0 ? "cycle_down_finest" : "cycle_down0_finest",
                          (double)L.cells * (v0 ? 12.0 : 8.0) + (double)C.cells * 4.0 + frac_bytes(L), s,
                          okl = launch_cycle_down(L, L.t, C.f, v0, (const float*)f, (float)w, zc, s));
                if (!okl) { wp_set_error_msg("fused cycle: no tensor map for the level"); return WP_ERR_CUDA; }
                std::swap(L.v, L.t);
                if ((st = vcycle<T>(h, l + 1, Bufs<T>::f(C), nu1, nu2, w, prolong, s, true)) != WP_OK) return st;
                const bool acc = acc64 != nullptr && added != nullptr && al16(acc64);
                WP_KERNEL(acc ? "cycle_up_update_finest" : "cycle_up_finest",
                          (double)L.cells * (acc ? 24.0 : 12.0) + (double)C.cells * 4.0 + frac_bytes(L), s,
                          okl = launch_cycle_up(L, C, acc ? nullptr : L.t, acc ? acc64 : nullptr, L.v, C.v,
                                                (const float*)f, (float)w, zc, s));
                if (!okl) { wp_set_error_msg("fused cycle: no tensor map for the level"); return WP_ERR_CUDA; }
                if (acc) *added = true;
                std::swap(L.v, L.t);
                return WP_OK;
            }
        }
        int pre = nu1;
        if (clear_v) {
            const int var = sizeof(T) == 4 ? L.var[kZcJacobi] : 0;
            if (nu1 > 0 && quad_ok(L) && al16(Bufs<T>::t(L)) && al16(f) && var != 3 && var != 4) {
                const int zc = level_zc(L, kZcJacobi);
                const dim3 gq(wp_cdiv((size_t)L.n[0] * (L.n[1] / 4), 256), wp_cdiv(L.n[2], zc));
                WP_KERNEL(l == 0 ? "jacobi0_finest" : "jacobi0", (double)L.cells * 2.0 * sizeof(T) + frac_bytes(L), s,
                          wp_launch_pdl(jacobi0_q_kernel<T>, gq, 256, 0, s, Bufs<T>::t(L), f, view<T>(L), w, zc));
                std::swap(Bufs<T>::v(L), Bufs<T>::t(L));
                pre = nu1 - 1;
            } else {
                WP_CUDA_TRY(cudaMemsetAsync(Bufs<T>::v(L), 0, sizeof(T) * L.cells, s));
            }
        }
        if ((st = smooth<T>(L, f, pre, w, s, l == 0)) != WP_OK) return st;
        Level& C = h->lv[l + 1];
        {
            // coarse-z chunk so the fine columns keep >= 4 CTAs per SM busy
            const int czc = level_zc(L, kZcRestrict);
            WP_KERNEL(l == 0 ? "resid_restrict_finest" : "resid_restrict",
                      (double)L.cells * 2.0 * sizeof(T) + frac_bytes(L) + (double)C.cells * sizeof(T), s,
                      launch_resid_restrict<T>(L, C, Bufs<T>::f(C), Bufs<T>::v(L), f, czc, s));
        }
        if ((st = vcycle<T>(h, l + 1, Bufs<T>::f(C), nu1, nu2, w, prolong, s, true)) != WP_OK) return st;
        if (prolong == WP_PROLONG_TRILINEAR) {
            WP_KERNEL(l == 0 ? "prolong_trilinear_finest" : "prolong_trilinear",
                      (double)L.cells * 2.0 * sizeof(T) + (double)C.cells * sizeof(T), s,
                      launch_prolong_tri<T>(L, C, Bufs<T>::v(L), Bufs<T>::v(C), s));
            if ((st = smooth<T>(L, f, nu2, w, s, l == 0, acc64, added)) != WP_OK) return st;
        } else if (nu2 > 0) {
            // first post-sweep reads v + P vc directly (prolongation fused into the sweep)
            const int zc = level_zc(L, kZcJacobi);
            WP_KERNEL("jacobi_prolong", (double)L.cells * (3.0 * sizeof(T) + 12.0) + (double)C.cells * sizeof(T), s,
                      jacobi_z_kernel<T, true><<<grid_z(L.n[0], L.n[1], L.n[2], zc), dim3(32, 8), 0, s>>>(
                          Bufs<T>::t(L), Bufs<T>::v(L), f, view<T>(L), w, Bufs<T>::v(C), C.n[0], C.n[1], zc));
            T* tmp = Bufs<T>::v(L);
            Bufs<T>::v(L) = Bufs<T>::t(L);
            Bufs<T>::t(L) = tmp;
            if ((st = smooth<T>(L, f, nu2 - 1, w, s, l == 0, acc64, added)) != WP_OK) return st;
        } else {
            WP_KERNEL("prolong_constant", (double)L.cells * 2.0 * sizeof(T) + (double)C.cells * sizeof(T), s,
                      prolong_add_kernel<T><<<g, dim3(32, 8), 0, s>>>(Bufs<T>::v(L), Bufs<T>::v(C), L.n[0], L.n[1],
                                                                     L.n[2], C.n[0], C.n[1]));
        }
    } else {
        if (clear_v) WP_CUDA_TRY(cudaMemsetAsync(Bufs<T>::v(L), 0, sizeof(T) * L.cells, s));
        if ((st = coarsest_solve<T>(h, L, f, w, s)) != WP_OK) return st;
    }
    return WP_OK;
}

// Full-multigrid start: the right-hand side restricted to every level (the residual restriction of
// a zero iterate), the coarsest level solved from zero, then on each finer level the prolonged
// coarser solution followed by one V-cycle.  Leaves the finest level's iterate in its v; costs
// about one V-cycle more than a V-cycle and replaces the first cycles from a zero start.
template <typename T>
wp_status fmg_start(wp_mgfrac3d* h, const T* f0, int nu1, int nu2, T w, int prolong, cudaStream_t s,
                    double* acc64 = nullptr, bool* added = nullptr) {
    wp_status st;
    for (int l = 0; l + 1 < h->nl; ++l) {
        Level& L = h->lv[l];
        Level& C = h->lv[l + 1];
        const T* fl = l == 0 ? f0 : Bufs<T>::f(L);
        WP_CUDA_TRY(cudaMemsetAsync(Bufs<T>::v(L), 0, sizeof(T) * L.cells, s));
        WP_KERNEL("fmg_restrict", (double)L.cells * (2.0 * sizeof(T) + 12.0) + (double)C.cells * sizeof(T), s,
                  launch_resid_restrict<T>(L, C, Bufs<T>::f(C), Bufs<T>::v(L), fl, level_zc(L, kZcRestrict), s));
    }
    const int lc = h->nl - 1;
    if ((st = vcycle<T>(h, lc, lc == 0 ? f0 : Bufs<T>::f(h->lv[lc]), nu1, nu2, w, prolong, s, true)) != WP_OK) return st;
    for (int l = lc - 1; l >= 0; --l) {
        Level& L = h->lv[l];
        Level& C = h->lv[l + 1];
        WP_CUDA_TRY(cudaMemsetAsync(Bufs<T>::v(L), 0, sizeof(T) * L.cells, s));
        if (prolong == WP_PROLONG_TRILINEAR)
            WP_KERNEL("fmg_prolong", (double)L.cells * 2.0 * sizeof(T) + (double)C.cells * sizeof(T), s,
                      launch_prolong_tri<T>(L, C, Bufs<T>::v(L), Bufs<T>::v(C), s));
        else
            WP_KERNEL("fmg_prolong", (double)L.cells * 2.0 * sizeof(T) + (double)C.cells * sizeof(T), s,
                      prolong_add_kernel<T><<<grid_of(L.n[0], L.n[1], L.n[2]), dim3(32, 8), 0, s>>>(
                          Bufs<T>::v(L), Bufs<T>::v(C), L.n[0], L.n[1], L.n[2], C.n[0], C.n[1]));
        if ((st = vcycle<T>(h, l, l == 0 ? f0 : Bufs<T>::f(L), nu1, nu2, w, prolong, s, false, l == 0 ? acc64 : nullptr,
                            l == 0 ? added : nullptr)) != WP_OK)
            return st;
    }
    return WP_OK;
}

// sum and count of f over the active cells of the level into acc[0], acc[1] (asynchronous)
void launch_active_sum(const Level& L, const float* f, double* acc, cudaStream_t s) {
    if (quad_ok(L) && al16(f)) {
        const int zc = std::max(1, std::min(L.n[2], 16));
        const dim3 g(wp_cdiv((size_t)L.n[0] * (L.n[1] / 4), 256), wp_cdiv(L.n[2], zc));
        active_sum_q_kernel<<<g, 256, 0, s>>>(f, view<double>(L), acc, zc);
    } else {
        active_sum_kernel<<<grid_of(L.n[0], L.n[1], L.n[2]), dim3(32, 8), 0, s>>>(f, view<double>(L), acc);
    }
}

// mean of f over the active cells of the finest level (synchronous)
wp_status active_mean(wp_mgfrac3d* h, const float* f, double* m, cudaStream_t s) {
    Level& L = h->lv[0];
    WP_CUDA_TRY(cudaMemsetAsync(h->acc + 2, 0, 2 * sizeof(double), s));
    WP_KERNEL("active_sum", (double)L.cells * 4.0 + frac_bytes(L), s, launch_active_sum(L, f, h->acc + 2, s));
    double hv[2];
    WP_CUDA_TRY(wp_read_small(hv, h->acc + 2, sizeof(hv), s));
    *m = hv[1] > 0 ? hv[0] / hv[1] : 0.0;
    return WP_OK;
}

// asynchronous FP64 defect: acc[0] = ||f - m - A p||^2 (msum: device mean slots, or NULL to use m),
// optionally acc[1] = ||f||^2
template <typename TP>
wp_status defect_async(wp_mgfrac3d* h, const TP* p, const float* f, double m, const double* msum, float* r32,
                       bool with_f2, cudaStream_t s) {
    Level& L = h->lv[0];
    WP_CUDA_TRY(cudaMemsetAsync(h->acc, 0, (with_f2 ? 2 : 1) * sizeof(double), s));
    const int zc = level_zc(L, kZcDefect);
    WP_KERNEL("defect64", (double)L.cells * (sizeof(TP) + 4.0 + (r32 ? 4.0 : 0.0)) + frac_bytes(L), s,
              launch_defect64<TP>(L, r32, p, f, m, msum, h->acc, zc, s));
    if (with_f2) {
        const unsigned b = std::min<unsigned>(wp_cdiv(L.cells, 256), wp_sm_count() * 8);
        WP_KERNEL("sumsq", 4.0 * L.cells, s, sumsq_kernel<float><<<b, 256, 0, s>>>(f, L.cells, h->acc + 1));
    }
    return WP_OK;
}

// Turns the handle's device error flag (a grid barrier or a pipeline wait that gave up) into a status,
// clearing it: the call that saw it fails with WP_ERR_DEVICE_WAIT, the handle stays usable.
wp_status device_wait_status(wp_mgfrac3d* h, int flag, cudaStream_t s) {
    if (!flag) return WP_OK;
    WP_CUDA_TRY(cudaMemsetAsync(h->acc + 4, 0, sizeof(int), s));
    wp_set_error_msg(flag & 2 ? "multigrid: a grid barrier wait gave up; the iterate of this call is invalid"
                              : "multigrid: a tile pipeline wait gave up; the iterate of this call is invalid");
    return WP_ERR_DEVICE_WAIT;
}

wp_status check_device_wait(wp_mgfrac3d* h, cudaStream_t s) {
    int flag = 0;
    WP_CUDA_TRY(wp_read_small(&flag, h->acc + 4, sizeof(int), s));
    return device_wait_status(h, flag, s);
}

template <typename TP>
wp_status defect(wp_mgfrac3d* h, const TP* p, const float* f, double m, float* r32, double* norm_r2,
                 double* norm_f2, cudaStream_t s) {
    Level& L = h->lv[0];
    WP_CUDA_TRY(cudaMemsetAsync(h->acc, 0, 2 * sizeof(double), s));
    const int zc = level_zc(L, kZcDefect);
    WP_KERNEL("defect64", (double)L.cells * (sizeof(TP) + 4.0 + (r32 ? 4.0 : 0.0)) + frac_bytes(L), s,
              launch_defect64<TP>(L, r32, p, f, m, nullptr, h->acc, zc, s));
    if (norm_f2) {
        const unsigned b = std::min<unsigned>(wp_cdiv(L.cells, 256), wp_sm_count() * 8);
        WP_KERNEL("sumsq", 4.0 * L.cells, s, sumsq_kernel<float><<<b, 256, 0, s>>>(f, L.cells, h->acc + 1));
    }
    // the two sums and, in the same read, the device error flag that follows the four slots
    struct {
        double v[4];
        int err;
    } hv;
    WP_CUDA_TRY(wp_read_small(&hv, h->acc, 4 * sizeof(double) + sizeof(int), s));
    *norm_r2 = hv.v[0];
    if (norm_f2) *norm_f2 = hv.v[1];
    return device_wait_status(h, hv.err, s);
}

void destroy_levels(wp_mgfrac3d* h) {
    for (int l = 0; l < kMaxLevels; ++l) {
        Level& L = h->lv[l];
        for (int a = 0; a < 3; ++a) if (L.frac[a]) cudaFree(L.frac[a]);
        void* ps[] = {L.tab64, L.tab32, L.fyc, L.uni, L.tuni, L.v, L.t, L.f, L.v64, L.t64, L.f64, L.imask, L.iseg};
        for (void* p : ps) if (p) cudaFree(p);
    }
    if (h->ccf_all) cudaFree(h->ccf_all);
    if (h->acc) cudaFree(h->acc);
    if (h->p64) cudaFree(h->p64);
    if (h->r32) cudaFree(h->r32);
    if (h->ix_r) cudaFree(h->ix_r);
    if (h->ix_r64) cudaFree(h->ix_r64);
}

wp_status create_common(wp_mgfrac3d** out, int dims, const float* ax, const float* ay, const float* az, int nx, int ny,
                        int nz, double dx, double dy, double dz, char bc, cudaStream_t s) {
    if (!out) { wp_set_error_msg("wp_mgfrac_create: null handle"); return WP_ERR_INVALID_ARG; }
    *out = nullptr;
    if (!ax || !ay || (dims == 3 && !az) || nx < 2 || ny < 2 || (dims == 3 && nz < 2) || nz > 65535 ||
        !(dx > 0) || !(dy > 0) || !(dz > 0)) {
        wp_set_error_msg("wp_mgfrac_create: bad arguments (extents >= 2, spacings > 0, fraction pointers)");
        return WP_ERR_INVALID_ARG;
    }
    if (bc != 'n') { wp_set_error_msg("wp_mgfrac_create: only bc 'n' (zero-flux walls) is implemented"); return WP_ERR_UNSUPPORTED; }
    wp_mgfrac3d* h = new (std::nothrow) wp_mgfrac3d();
    if (!h) return WP_ERR_INVALID_ARG;
    h->dims = dims;
    h->coarsest_iters = dims == 3 ? 50 : 10;
    h->mid_on = 1;
    h->fz_on = 1;
    wp_status st = build_hierarchy(h, ax, ay, az, nx, ny, nz, dx, dy, dz, s);
    if (st == WP_OK) {
        cudaError_t e = cudaMalloc((void**)&h->acc, 4 * sizeof(double) + 16);
        // the int error flag lives in the 16 bytes after the four FP64 slots
        if (e == cudaSuccess) e = cudaMemsetAsync(h->acc, 0, 4 * sizeof(double) + 16, s);
        if (e == cudaSuccess)
            for (int l = 0; l < h->nl; ++l) h->lv[l].err = reinterpret_cast<int*>(h->acc + 4);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { wp_set_cuda_error(e, "mg create", __FILE__, __LINE__); st = WP_ERR_CUDA; }
    }
    if (st != WP_OK) { destroy_levels(h); delete h; return st; }
    *out = h;
    return WP_OK;
}

wp_status solve_fixed(wp_mgfrac3d* h, float* dst, const float* pre_v, const float* f, int n_iters, int nu1, int nu2,
                      double weight, cudaStream_t s) {
    if (!h || !dst || !f || n_iters < 0 || nu1 < 0 || nu2 < 0) { wp_set_error_msg("wp_mgfrac_solve: bad arguments"); return WP_ERR_INVALID_ARG; }
    Level& L = h->lv[0];
    if (pre_v) WP_CUDA_TRY(cudaMemcpyAsync(L.v, pre_v, sizeof(float) * L.cells, cudaMemcpyDeviceToDevice, s));
    else WP_CUDA_TRY(cudaMemsetAsync(L.v, 0, sizeof(float) * L.cells, s));
    for (int c = 0; c < n_iters; ++c) {
        wp_status st = vcycle<float>(h, 0, f, nu1, nu2, (float)weight, WP_PROLONG_CONSTANT, s, false);
        if (st != WP_OK) return st;
    }
    WP_CUDA_TRY(cudaMemcpyAsync(dst, L.v, sizeof(float) * L.cells, cudaMemcpyDeviceToDevice, s));
    return check_device_wait(h, s);
}

// The index lists of every level (InitIndex, cuMultigridFrac3D.cu:189-229) and the zeroed residual
// workspace; once per handle, synchronous (the list lengths size the launches).
wp_status build_index(wp_mgfrac3d* h, cudaStream_t s) {
    if (h->ix_built) return WP_OK;
    long maxseg = 0;
    for (int l = 0; l < h->nl; ++l) {
        const Level& L = h->lv[l];
        maxseg = std::max(maxseg, (long)L.n[0] * L.n[2] * (long)wp_cdiv(L.n[1], 32));
    }
    const long maxb = (long)wp_cdiv(maxseg, kIxBlock);
    int* bcount = nullptr;
    long long* dev = nullptr;  // [0] listed segments, [1] selected cells
    wp_status st = WP_OK;
    auto fail = [&](cudaError_t e, int line) {
        wp_set_cuda_error(e, "index lists", __FILE__, line);
        st = WP_ERR_CUDA;
    };
    cudaError_t e = cudaMalloc((void**)&bcount, sizeof(int) * maxb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&dev, 2 * sizeof(long long));
    if (e != cudaSuccess) fail(e, __LINE__);
    for (int l = 0; l < h->nl && st == WP_OK; ++l) {
        Level& L = h->lv[l];
        const int nsy = (int)wp_cdiv(L.n[1], 32);
        const long nseg = (long)L.n[0] * L.n[2] * nsy;
        const int nb = (int)wp_cdiv(nseg, kIxBlock);
        if (L.imask) cudaFree(L.imask);
        if (L.iseg) cudaFree(L.iseg);
        L.imask = nullptr;
        L.iseg = nullptr;
        e = cudaMalloc((void**)&L.imask, sizeof(unsigned) * nseg);
        if (e == cudaSuccess) e = cudaMemsetAsync(dev, 0, 2 * sizeof(long long), s);
        if (e != cudaSuccess) { fail(e, __LINE__); break; }
        WP_KERNEL("index_mask", 12.0 * L.cells, s,
                  index_mask_kernel<<<(unsigned)wp_cdiv(nseg * 32, 256), 256, 0, s>>>(
                      L.imask, reinterpret_cast<unsigned long long*>(dev + 1), view<float>(L), nsy, nseg));
        WP_KERNEL("index_count", 4.0 * nseg, s, index_count_kernel<<<nb, kIxBlock, 0, s>>>(L.imask, nseg, bcount));
        WP_KERNEL("index_scan", 8.0 * nb, s, index_scan_kernel<<<1, 1024, 0, s>>>(bcount, nb, dev));
        long long hv[2] = {0, 0};
        e = cudaMemcpyAsync(hv, dev, sizeof(hv), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { fail(e, __LINE__); break; }
        L.iseg_n = hv[0];
        L.icells = hv[1];
        if (hv[0] > 0) {
            e = cudaMalloc((void**)&L.iseg, sizeof(int4) * hv[0]);
            if (e != cudaSuccess) { fail(e, __LINE__); break; }
            WP_KERNEL("index_scatter", 4.0 * nseg + 16.0 * hv[0], s,
                      index_scatter_kernel<<<nb, kIxBlock, 0, s>>>(L.imask, nseg, bcount, L.iseg, nsy, L.n[0]));
        }
    }
    if (st == WP_OK) {
        if (h->ix_r) cudaFree(h->ix_r);
        h->ix_r = nullptr;
        e = cudaMalloc((void**)&h->ix_r, sizeof(float) * h->lv[0].cells);
        if (e == cudaSuccess) e = cudaMemsetAsync(h->ix_r, 0, sizeof(float) * h->lv[0].cells, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) fail(e, __LINE__);
    }
    if (bcount) cudaFree(bcount);
    if (dev) cudaFree(dev);
    if (st == WP_OK) h->ix_built = 1;
    return st;
}

// One index-sparse V-cycle at level l (SolveOneVCycle_index, cuMultigridFrac3D.cu:366-420).  A
// coarse level enters with v = 0 at every cell: its unlisted cells stay 0 throughout the solve (no
// index kernel writes them) and its first sweep computes the listed ones from zero.  The cycle goes
// down while the next level lists a cell, then the coarsest solve runs; post-smoothing runs nu1
// sweeps, as the reference passes nu1 there.  r: the residual workspace (finest size).
template <typename T>
wp_status vcycle_ix(wp_mgfrac3d* h, int l, const T* f, T* r, int nu1, T w, cudaStream_t s) {
    Level& L = h->lv[l];
    T*& v = Bufs<T>::v(L);
    T*& t = Bufs<T>::t(L);
    if (!(l < h->nl - 1 && h->lv[l + 1].icells > 0)) {
        if (l > 0) WP_CUDA_TRY(cudaMemsetAsync(v, 0, sizeof(T) * L.cells, s));
        return coarsest_solve<T>(h, L, f, w, s);
    }
    Level& C = h->lv[l + 1];
    const unsigned gb = (unsigned)wp_cdiv(L.iseg_n, 8), gc = (unsigned)wp_cdiv(C.iseg_n, 8);
    const double lc = (double)L.icells, ls = (double)L.iseg_n, B = sizeof(T);
    const int4* seg = L.iseg;
    const long nseg = (long)L.iseg_n;
    auto sweeps = [&](bool first_from_zero) -> wp_status {
        for (int k = 0; k < nu1; ++k) {
            if (gb > 0) {
                if (k == 0 && first_from_zero && l > 0)
                    WP_KERNEL("jacobi0_ix", lc * (2.0 * B + 12.0) + 16.0 * ls, s,
                              wp_launch_pdl(jacobi0_ix_kernel<T>, gb, 256, 0, s, t, f, view<T>(L), w, seg, nseg));
                else
                    WP_KERNEL(l == 0 ? "jacobi_ix_finest" : "jacobi_ix", lc * (3.0 * B + 12.0) + 16.0 * ls, s,
                              wp_launch_pdl(jacobi_ix_kernel<T>, gb, 256, 0, s, t, (const T*)v, f, view<T>(L), w,
                                            seg, nseg));
            }
            std::swap(v, t);
        }
        return WP_OK;
    };
    wp_status st;
    if (l > 0 && nu1 == 0) WP_CUDA_TRY(cudaMemsetAsync(v, 0, sizeof(T) * L.cells, s));
    if ((st = sweeps(true)) != WP_OK) return st;
    if (gb > 0)
        WP_KERNEL(l == 0 ? "resid_ix_finest" : "resid_ix", lc * (3.0 * B + 12.0) + 16.0 * ls, s,
                  wp_launch_pdl(resid_ix_kernel<T>, gb, 256, 0, s, r, (const T*)v, f, view<T>(L), seg, nseg));
    // the coarsest solve sweeps every cell of its level: the unlisted ones read a zero right-hand
    // side (the reference's never-written coarse arrays; they matter where a face fraction is
    // nonzero but below the selection threshold)
    if (!(l + 1 < h->nl - 1 && h->lv[l + 2].icells > 0))
        WP_CUDA_TRY(cudaMemsetAsync(Bufs<T>::f(C), 0, sizeof(T) * C.cells, s));
    if (gc > 0)
        WP_KERNEL("restrict_ix", (double)C.icells * (9.0 * B) + 16.0 * C.iseg_n, s,
                  wp_launch_pdl(restrict_ix_kernel<T>, gc, 256, 0, s, Bufs<T>::f(C), (const T*)r, view<T>(L), C.n[0],
                                C.n[1], (const int4*)C.iseg, (long)C.iseg_n));
    if ((st = vcycle_ix<T>(h, l + 1, Bufs<T>::f(C), r, nu1, w, s)) != WP_OK) return st;
    // a separate pass: folding the prolongation into the first post-sweep needs the neighbours'
    // selection bits and parent values as dependent loads, which measured slower (117 against
    // 25 + 51 us at 256^3, 15% fluid)
    if (gb > 0)
        WP_KERNEL(l == 0 ? "prolong_ix_finest" : "prolong_ix", lc * (3.0 * B) + 16.0 * ls, s,
                  wp_launch_pdl(prolong_ix_kernel<T>, gb, 256, 0, s, v, (const T*)Bufs<T>::v(C), view<T>(L), C.n[0],
                                C.n[1], seg, nseg));
    return sweeps(false);
}

// CuMultigridFrac3D::Solve_index (cuMultigridFrac3D.cu:347-364): n_iters index-sparse V-cycles in T.
// The finest level's unlisted cells keep their start value (pre_v, or 0).
template <typename T>
wp_status solve_index(wp_mgfrac3d* h, T* dst, const T* pre_v, const T* f, int n_iters, int nu1, int nu2,
                      double weight, cudaStream_t s) {
    if (!h || !dst || !f || n_iters < 0 || nu1 < 0 || nu2 < 0) {
        wp_set_error_msg("wp_mgfrac3d_solve_index: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    if (h->dims != 3) {
        wp_set_error_msg("wp_mgfrac3d_solve_index: the index-sparse cycle is 3D only");
        return WP_ERR_UNSUPPORTED;
    }
    wp_status st = build_index(h, s);
    if (st != WP_OK) return st;
    T* r = nullptr;
    if (sizeof(T) == 4) {
        r = reinterpret_cast<T*>(h->ix_r);
    } else {
        if ((st = ensure_fp64(h)) != WP_OK) return st;
        if (!h->ix_r64) {
            WP_CUDA_TRY(cudaMalloc((void**)&h->ix_r64, sizeof(double) * h->lv[0].cells));
            WP_CUDA_TRY(cudaMemsetAsync(h->ix_r64, 0, sizeof(double) * h->lv[0].cells, s));
        }
        r = reinterpret_cast<T*>(h->ix_r64);
    }
    Level& L = h->lv[0];
    T* v = Bufs<T>::v(L);
    if (pre_v) WP_CUDA_TRY(cudaMemcpyAsync(v, pre_v, sizeof(T) * L.cells, cudaMemcpyDeviceToDevice, s));
    else WP_CUDA_TRY(cudaMemsetAsync(v, 0, sizeof(T) * L.cells, s));
    WP_CUDA_TRY(cudaMemcpyAsync(Bufs<T>::t(L), v, sizeof(T) * L.cells, cudaMemcpyDeviceToDevice, s));
    for (int l = 1; l < h->nl; ++l) {
        WP_CUDA_TRY(cudaMemsetAsync(Bufs<T>::v(h->lv[l]), 0, sizeof(T) * h->lv[l].cells, s));
        WP_CUDA_TRY(cudaMemsetAsync(Bufs<T>::t(h->lv[l]), 0, sizeof(T) * h->lv[l].cells, s));
    }
    for (int c = 0; c < n_iters; ++c)
        if ((st = vcycle_ix<T>(h, 0, f, r, nu1, (T)weight, s)) != WP_OK) return st;
    WP_CUDA_TRY(cudaMemcpyAsync(dst, Bufs<T>::v(L), sizeof(T) * L.cells, cudaMemcpyDeviceToDevice, s));
    // the FP64 level buffers held the last FP64 tolerance solve's iterate: it is gone
    if (sizeof(T) == 8 && h->last64 == 2) h->last64 = 0;
    return WP_OK;
}

int inner_of(const wp_mg_params* prm) { return prm->inner_cycles > 1 ? prm->inner_cycles : 1; }

// The correction of one refinement step of the mixed solve: inner_cycles FP32 V-cycles on
// A e = r32 (the first from e = 0, or a full-multigrid start), then p64 += e -- fused into the
// last post-sweep where the level's kernel allows, add_correction_kernel otherwise.
wp_status mixed_correction(wp_mgfrac3d* h, const wp_mg_params* prm, bool fmg, cudaStream_t s) {
    Level& L = h->lv[0];
    const long n = L.cells;
    const int inner = inner_of(prm);
    bool added = false;
    for (int j = 0; j < inner; ++j) {
        double* acc = j == inner - 1 ? h->p64 : nullptr;
        bool* ad = j == inner - 1 ? &added : nullptr;
        wp_status st;
        if (j == 0 && fmg)
            st = fmg_start<float>(h, h->r32, prm->nu1, prm->nu2, (float)prm->omega, prm->prolongation, s, acc, ad);
        else
            st = vcycle<float>(h, 0, h->r32, prm->nu1, prm->nu2, (float)prm->omega, prm->prolongation, s, j == 0, acc,
                               ad);
        if (st != WP_OK) return st;
    }
    if (!added) {
        const unsigned cb = std::min<unsigned>(wp_cdiv(n, 256), wp_sm_count() * 8);
        WP_KERNEL("add_correction", 20.0 * n, s,
                  wp_launch_pdl(add_correction_kernel, cb, 256, 0, s, h->p64, (const float*)L.v, n));
    }
    return WP_OK;
}

// State of the device-side cycle loop: the stopping rule of solve_tol's host loop, evaluated by
// mg_loop_check_kernel after every defect (cycles advance by `inner` per refinement step).
struct MgLoop {
    int cycles, max_cycles, use_tol, inner, steps, pad;
    double tol, rel;
    double hist[64];
};

__global__ void mg_loop_init_kernel(MgLoop* st, int max_cycles, int use_tol, double tol, int inner) {
    st->cycles = 0;
    st->steps = 0;
    st->max_cycles = max_cycles;
    st->use_tol = use_tol;
    st->inner = inner;
    st->tol = tol;
    st->rel = 0.0;
}

// rel = sqrt(||r||^2 / ||f||^2) of the defect just computed (acc[0], acc[1]; ||f|| = 0 counts as 1),
// recorded as in solve_tol; the loop goes on while the tolerance is not met, the cycle cap not
// reached and rel is finite
__global__ void mg_loop_check_kernel(MgLoop* st, const double* __restrict__ acc, cudaGraphConditionalHandle hc) {
    wp_pdl_enter();
    double nf2 = acc[1];
    if (!(nf2 > 0.0)) nf2 = 1.0;
    const double rel = sqrt(acc[0] / nf2);
    const int k = st->steps, c = st->cycles + st->inner;
    if (k < 64) st->hist[k] = rel;
    st->steps = k + 1;
    st->cycles = c;
    st->rel = rel;
    const bool go = !(st->use_tol && rel <= st->tol) && c < st->max_cycles && isfinite(rel);
    cudaGraphSetConditional(hc, go ? 1u : 0u);
}

void destroy_loop_graph(wp_mgfrac3d* h) {
    if (h->loop_exec) cudaGraphExecDestroy(h->loop_exec);
    if (h->loop_graph) cudaGraphDestroy(h->loop_graph);
    h->loop_exec = nullptr;
    h->loop_graph = nullptr;
    h->loop_f = nullptr;
}

// one refinement step of the mixed solve on the device: FP32 correction cycle on r32 (the first
// one a full-multigrid start if fmg), FP64 update, FP64 defect with the device mean, loop test
wp_status mixed_step(wp_mgfrac3d* h, const float* f, const wp_mg_params* prm, bool fmg, cudaGraphConditionalHandle hc,
                     cudaStream_t s) {
    wp_status st;
    if ((st = mixed_correction(h, prm, fmg, s)) != WP_OK) return st;
    if ((st = defect_async<double>(h, h->p64, f, 0.0, h->acc + 2, h->r32, false, s)) != WP_OK) return st;
    WP_KERNEL("mg_loop_check", 0.0, s,
              wp_launch_pdl(mg_loop_check_kernel, 1, 1, 0, s, (MgLoop*)h->loop_state, (const double*)h->acc, hc));
    return WP_OK;
}

// Builds the graph [first step] -> while (go) [step]: the first step is captured into the parent
// graph, a while-node on the condition the check kernels set follows it, and one step is captured
// into the node's body.  Every buffer a step reads is written earlier in the same step or is
// loop-invariant (r32, p64, acc, f), so replaying the body repeats the host loop exactly.
wp_status build_loop_graph(wp_mgfrac3d* h, const float* f, const wp_mg_params* prm, bool fmg) {
    destroy_loop_graph(h);
    if (!h->loop_state) WP_CUDA_TRY(cudaMalloc(&h->loop_state, sizeof(MgLoop)));
    if (!h->loop_cap) WP_CUDA_TRY(cudaStreamCreateWithFlags(&h->loop_cap, cudaStreamNonBlocking));
    cudaStream_t s = h->loop_cap;
    cudaGraph_t g = nullptr;
    WP_CUDA_TRY(cudaGraphCreate(&g, 0));
    h->loop_graph = g;
    cudaGraphConditionalHandle hc;
    WP_CUDA_TRY(cudaGraphConditionalHandleCreate(&hc, g, 0, cudaGraphCondAssignDefault));
    const long long c0 = wp_launch_count();
    WP_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    wp_status st = mixed_step(h, f, prm, fmg, hc, s);
    cudaGraphNode_t cn = nullptr;
    cudaError_t e = cudaSuccess;
    if (st == WP_OK) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd);
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = hc;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        if (e == cudaSuccess) e = cudaGraphAddNode(&cn, cg, deps, nd, &cp);
        if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(s, &cn, 1, cudaStreamSetCaptureDependencies);
        if (e == cudaSuccess) {
            cudaGraph_t out = nullptr;
            e = cudaStreamEndCapture(s, &out);
            const long long c1 = wp_launch_count();
            if (e == cudaSuccess) {
                cudaGraph_t body = cp.conditional.phGraph_out[0];
                e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
                if (e == cudaSuccess) {
                    st = mixed_step(h, f, prm, false, hc, s);
                    cudaGraph_t bout = nullptr;
                    const cudaError_t e2 = cudaStreamEndCapture(s, &bout);
                    if (st == WP_OK) e = e2;
                }
            }
            h->loop_launches[0] = c1 - c0;
            h->loop_launches[1] = wp_launch_count() - c1;
        }
    }
    if (e != cudaSuccess || st != WP_OK) {
        // leave the stream out of capture mode whatever failed
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
            cudaGraph_t junk = nullptr;
            cudaStreamEndCapture(s, &junk);
        }
        (void)cudaGetLastError();
    }
    wp_add_launches(-(wp_launch_count() - c0));
    if (st != WP_OK) { destroy_loop_graph(h); return st; }
    if (e != cudaSuccess) { destroy_loop_graph(h); wp_set_cuda_error(e, "multigrid loop capture", __FILE__, __LINE__); return WP_ERR_CUDA; }
    e = cudaGraphInstantiate(&h->loop_exec, g, 0);
    if (e != cudaSuccess) { destroy_loop_graph(h); wp_set_cuda_error(e, "multigrid loop instantiate", __FILE__, __LINE__); return WP_ERR_CUDA; }
    int dev = 0;
    cudaGetDevice(&dev);
    h->loop_f = f;
    const int key[7] = {prm->nu1, prm->nu2, prm->prolongation, fmg ? 1 : 0, h->tune_gen, dev, inner_of(prm)};
    memcpy(h->loop_key, key, sizeof(key));
    h->loop_omega = prm->omega;
    return WP_OK;
}

bool loop_graph_ready(const wp_mgfrac3d* h, const float* f, const wp_mg_params* prm, bool fmg) {
    int dev = 0;
    cudaGetDevice(&dev);
    const int key[7] = {prm->nu1, prm->nu2, prm->prolongation, fmg ? 1 : 0, h->tune_gen, dev, inner_of(prm)};
    return h->loop_exec && h->loop_f == f && memcmp(key, h->loop_key, sizeof(key)) == 0 && h->loop_omega == prm->omega;
}

// The cycle loop of the mixed tolerance solve as one graph launch (the rest of solve_tol's mixed
// branch is unchanged): the same steps, stopping rule and report as the host loop, read back once.
wp_status solve_mixed_graph(wp_mgfrac3d* h, const float* f, const wp_mg_params* prm, bool fmg, wp_mg_report* r,
                            cudaStream_t s) {
    if (!loop_graph_ready(h, f, prm, fmg)) {
        wp_status st = build_loop_graph(h, f, prm, fmg);
        if (st != WP_OK) return st;
    }
    WP_KERNEL("mg_loop_init", 0.0, s,
              mg_loop_init_kernel<<<1, 1, 0, s>>>((MgLoop*)h->loop_state, prm->max_cycles, prm->rel_tol > 0.0 ? 1 : 0,
                                                  prm->rel_tol, inner_of(prm)));
    WP_CUDA_TRY(cudaGraphLaunch(h->loop_exec, s));
    MgLoop out;
    WP_CUDA_TRY(wp_read_small(&out, h->loop_state, sizeof(out), s));
    wp_add_launches(h->loop_launches[0] + (long long)(out.steps > 0 ? out.steps - 1 : 0) * h->loop_launches[1]);
    r->cycles = out.cycles;
    r->steps = out.steps;
    for (int c = 0; c < out.steps && c < 64; ++c) r->history[c] = out.hist[c];
    r->rel_residual = out.rel;
    return WP_OK;
}

wp_status solve_tol(wp_mgfrac3d* h, float* dst, const float* pre_v, const float* f, const wp_mg_params* prm,
                    wp_mg_report* rep, cudaStream_t s) {
    if (!h || !dst || !f || !prm || prm->max_cycles < 0 || prm->nu1 < 0 || prm->nu2 < 0 ||
        (prm->prolongation != WP_PROLONG_CONSTANT && prm->prolongation != WP_PROLONG_TRILINEAR)) {
        wp_set_error_msg("wp_mgfrac_solve_tol: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    Level& L = h->lv[0];
    const long n = L.cells;
    const unsigned cb = std::min<unsigned>(wp_cdiv(n, 256), wp_sm_count() * 8);
    wp_mg_report r;
    memset(&r, 0, sizeof(r));
    double nr2 = 0.0, nf2 = 0.0, m = 0.0;
    wp_status st = active_mean(h, f, &m, s);
    if (st != WP_OK) return st;
    const bool use_tol = prm->rel_tol > 0.0;
    if (prm->precision == WP_PREC_FP32 || prm->precision == WP_PREC_FP64) {
        const bool f64 = prm->precision == WP_PREC_FP64;
        if (f64) {
            if ((st = ensure_fp64(h)) != WP_OK) return st;
            WP_KERNEL("rhs64", 28.0 * n, s,
                      rhs64_kernel<<<grid_of(L.n[0], L.n[1], L.n[2]), dim3(32, 8), 0, s>>>(L.f64, f, view<double>(L), m));
            if (pre_v) WP_KERNEL("convert", 12.0 * n, s, convert_kernel<double, float><<<cb, 256, 0, s>>>(L.v64, pre_v, n));
            else WP_CUDA_TRY(cudaMemsetAsync(L.v64, 0, sizeof(double) * n, s));
        } else {
            if (pre_v) WP_CUDA_TRY(cudaMemcpyAsync(L.v, pre_v, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
            else WP_CUDA_TRY(cudaMemsetAsync(L.v, 0, sizeof(float) * n, s));
        }
        if (f64) st = defect<double>(h, L.v64, f, m, nullptr, &nr2, &nf2, s);
        else st = defect<float>(h, L.v, f, m, nullptr, &nr2, &nf2, s);
        if (st != WP_OK) return st;
        if (!(nf2 > 0.0)) nf2 = 1.0;
        double rel = std::sqrt(nr2 / nf2);
        while (!(use_tol && rel <= prm->rel_tol) && r.cycles < prm->max_cycles) {
            const bool fmg = r.cycles == 0 && !pre_v && prm->start == WP_START_FMG;
            if (fmg)
                st = f64 ? fmg_start<double>(h, L.f64, prm->nu1, prm->nu2, prm->omega, prm->prolongation, s)
                         : fmg_start<float>(h, f, prm->nu1, prm->nu2, (float)prm->omega, prm->prolongation, s);
            else
                st = f64 ? vcycle<double>(h, 0, L.f64, prm->nu1, prm->nu2, prm->omega, prm->prolongation, s, false)
                         : vcycle<float>(h, 0, f, prm->nu1, prm->nu2, (float)prm->omega, prm->prolongation, s, false);
            if (st != WP_OK) return st;
            if (f64) st = defect<double>(h, L.v64, f, m, nullptr, &nr2, nullptr, s);
            else st = defect<float>(h, L.v, f, m, nullptr, &nr2, nullptr, s);
            if (st != WP_OK) return st;
            rel = std::sqrt(nr2 / nf2);
            if (r.cycles < 64) r.history[r.cycles] = rel;
            r.steps = ++r.cycles;
            if (!std::isfinite(rel)) break;
        }
        r.rel_residual = rel;
        h->last64 = f64 ? 2 : 0;
        if (f64) WP_KERNEL("convert", 12.0 * n, s, convert_kernel<float, double><<<cb, 256, 0, s>>>(dst, L.v64, n));
        else WP_CUDA_TRY(cudaMemcpyAsync(dst, L.v, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
    } else if (prm->precision == WP_PREC_MIXED) {
        if (!h->p64) WP_CUDA_TRY(cudaMalloc((void**)&h->p64, sizeof(double) * n));
        if (!h->r32) WP_CUDA_TRY(cudaMalloc((void**)&h->r32, sizeof(float) * n));
        if (pre_v) WP_KERNEL("convert", 12.0 * n, s, convert_kernel<double, float><<<cb, 256, 0, s>>>(h->p64, pre_v, n));
        else WP_CUDA_TRY(cudaMemsetAsync(h->p64, 0, sizeof(double) * n, s));
        if ((st = defect<double>(h, h->p64, f, m, h->r32, &nr2, &nf2, s)) != WP_OK) return st;
        if (!(nf2 > 0.0)) nf2 = 1.0;
        double rel = std::sqrt(nr2 / nf2);
        const bool go = !(use_tol && rel <= prm->rel_tol) && prm->max_cycles > 0;
        bool on_device = false;
        if (go && !prm->host_loop && !h->loop_broken && !wp_profile_is_enabled()) {
            // per-kernel timing events need the host loop; everything else runs the device loop
            const bool fmg = !pre_v && prm->start == WP_START_FMG;
            if (!loop_graph_ready(h, f, prm, fmg)) {
                // a driver without conditional graph nodes, or a failed capture: keep the host loop
                if (build_loop_graph(h, f, prm, fmg) != WP_OK) h->loop_broken = 1;
                (void)cudaGetLastError();
            }
            if (!h->loop_broken) {
                if ((st = solve_mixed_graph(h, f, prm, fmg, &r, s)) != WP_OK) return st;
                rel = r.rel_residual;
                on_device = true;
            }
        }
        int steps = 0;
        while (!on_device && !(use_tol && rel <= prm->rel_tol) && r.cycles < prm->max_cycles) {
            // one refinement step: FP32 correction cycles (the first one a full-multigrid start if
            // asked) on the FP32 defect, FP64 update, FP64 defect
            if ((st = mixed_correction(h, prm, r.cycles == 0 && !pre_v && prm->start == WP_START_FMG, s)) != WP_OK)
                return st;
            if ((st = defect<double>(h, h->p64, f, m, h->r32, &nr2, nullptr, s)) != WP_OK) return st;
            rel = std::sqrt(nr2 / nf2);
            if (steps < 64) r.history[steps] = rel;
            r.steps = ++steps;
            r.cycles += inner_of(prm);
            if (!std::isfinite(rel)) break;
        }
        r.rel_residual = rel;
        h->last64 = 1;
        WP_KERNEL("convert", 12.0 * n, s, convert_kernel<float, double><<<cb, 256, 0, s>>>(dst, h->p64, n));
    } else {
        wp_set_error_msg("wp_mgfrac_solve_tol: unknown precision mode");
        return WP_ERR_INVALID_ARG;
    }
    if (rep) *rep = r;
    if ((st = check_device_wait(h, s)) != WP_OK) return st;
    if (!std::isfinite(r.rel_residual)) { wp_set_error_msg("multigrid: non-finite residual"); return WP_ERR_NONFINITE; }
    if (use_tol && r.rel_residual > prm->rel_tol) { wp_set_error_msg("multigrid: cycle cap reached before tolerance"); return WP_ERR_NOT_CONVERGED; }
    return WP_OK;
}

// Allocates the mixed-precision work arrays ahead of a graph capture.
wp_status prepare_mixed(wp_mgfrac3d* h) {
    const long n = h->lv[0].cells;
    if (!h->p64) WP_CUDA_TRY(cudaMalloc((void**)&h->p64, sizeof(double) * n));
    if (!h->r32) WP_CUDA_TRY(cudaMalloc((void**)&h->r32, sizeof(float) * n));
    if (!h->loop_state) WP_CUDA_TRY(cudaMalloc(&h->loop_state, sizeof(MgLoop)));
    if (!h->loop_cap) WP_CUDA_TRY(cudaStreamCreateWithFlags(&h->loop_cap, cudaStreamNonBlocking));
    return WP_OK;
}

// The loop test before the first step (nothing counted): go while the initial defect misses the
// tolerance, the cycle cap allows a step and the residual is finite -- solve_tol's host test.
__global__ void mg_loop_start_kernel(MgLoop* st, const double* __restrict__ acc, cudaGraphConditionalHandle hc) {
    double nf2 = acc[1];
    if (!(nf2 > 0.0)) nf2 = 1.0;
    const double rel = sqrt(acc[0] / nf2);
    st->rel = rel;
    const bool go = !(st->use_tol && rel <= st->tol) && st->max_cycles > 0 && isfinite(rel);
    cudaGraphSetConditional(hc, go ? 1u : 0u);
}

// The tolerance-driven mixed solve with its cycle loop on the device, emitted into the graph the
// caller is capturing on s (a batch branch): the initial defect, a test kernel, then a while-node
// whose body is one refinement step ending in mg_loop_check_kernel, then dst = (float) p64.  Every
// replay re-runs the stopping rule of solve_tol on the current f, so the step count follows the
// input.  A full-multigrid start puts the first step before the loop, as the single-grid loop graph
// does.  *body_launches: kernels in one pass of the loop body.
wp_status solve_mixed_loop_capture(wp_mgfrac3d* h, float* dst, const float* f, const wp_mg_params* prm, cudaStream_t s,
                                   long long* body_launches) {
    Level& L = h->lv[0];
    const long n = L.cells;
    const unsigned cb = std::min<unsigned>(wp_cdiv(n, 256), wp_sm_count() * 8);
    wp_status st;
    if (!h->p64 || !h->r32 || !h->loop_state || !h->loop_cap) {
        wp_set_error_msg("mixed solve: work arrays not prepared");
        return WP_ERR_INVALID_ARG;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t cg = nullptr;
    WP_CUDA_TRY(cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, nullptr, nullptr));
    if (cs != cudaStreamCaptureStatusActive) {
        wp_set_error_msg("mixed solve loop: the stream is not capturing");
        return WP_ERR_INVALID_ARG;
    }
    cudaGraphConditionalHandle hc;
    WP_CUDA_TRY(cudaGraphConditionalHandleCreate(&hc, cg, 0, cudaGraphCondAssignDefault));
    WP_CUDA_TRY(cudaMemsetAsync(h->acc + 2, 0, 2 * sizeof(double), s));
    WP_KERNEL("active_sum", (double)n * 4.0 + frac_bytes(L), s, launch_active_sum(L, f, h->acc + 2, s));
    WP_CUDA_TRY(cudaMemsetAsync(h->p64, 0, sizeof(double) * n, s));
    if ((st = defect_async<double>(h, h->p64, f, 0.0, h->acc + 2, h->r32, true, s)) != WP_OK) return st;
    WP_KERNEL("mg_loop_init", 0.0, s,
              mg_loop_init_kernel<<<1, 1, 0, s>>>((MgLoop*)h->loop_state, prm->max_cycles, prm->rel_tol > 0.0 ? 1 : 0,
                                                  prm->rel_tol, inner_of(prm)));
    if (prm->start == WP_START_FMG) {
        if ((st = mixed_step(h, f, prm, true, hc, s)) != WP_OK) return st;
    } else {
        WP_KERNEL("mg_loop_start", 0.0, s,
                  mg_loop_start_kernel<<<1, 1, 0, s>>>((MgLoop*)h->loop_state, (const double*)h->acc, hc));
    }
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    WP_CUDA_TRY(cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = hc;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cn = nullptr;
    WP_CUDA_TRY(cudaGraphAddNode(&cn, cg, deps, nd, &cp));
    WP_CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &cn, 1, cudaStreamSetCaptureDependencies));
    // the body: one refinement step, captured on the handle's private stream into the node's graph
    const long long c0 = wp_launch_count();
    WP_CUDA_TRY(cudaStreamBeginCaptureToGraph(h->loop_cap, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal));
    st = mixed_step(h, f, prm, false, hc, h->loop_cap);
    cudaGraph_t bout = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->loop_cap, &bout);
    if (body_launches) *body_launches = wp_launch_count() - c0;
    wp_add_launches(-(wp_launch_count() - c0));  // counted per pass when the batch reads its results
    if (st != WP_OK) return st;
    if (e != cudaSuccess) { wp_set_cuda_error(e, "mixed solve loop body capture", __FILE__, __LINE__); return WP_ERR_CUDA; }
    h->last64 = 1;
    WP_KERNEL("convert", 12.0 * n, s, convert_kernel<float, double><<<cb, 256, 0, s>>>(dst, h->p64, n));
    return WP_OK;
}

// ---- persistent batched solve ------------------------------------------------------------------
// The mixed-precision tolerance solves of many grids in one persistent launch: one 1024-thread CTA
// per SM takes work from a queue until every grid's solve has ended.  Each grid's solve is a
// program of phases -- the launches of the launch-by-launch path: the active-cell sum with the FP64
// iterate cleared, the first FP64 defect with the start test, then one refinement step (inner V(nu1,
// nu2) cycles: first sweep from zero, sweeps, residual restriction, the single-CTA coarse cycle,
// trilinear prolongation, and the last post-sweep adding to the FP64 iterate), the FP64 defect with
// the stopping rule, and the FP32 copy of the solution.  The rule sends the program back to the
// step or on to the copy.  A phase is cut into tiles of the quad kernels' 256-thread blocks, run by
// the CTA's four 256-thread sub-blocks with every load of data written earlier in the launch taken
// through L2; the coarse cycle is one tile for the whole CTA.  Per grid one 64-bit word {phase,
// its tiles, next tile} hands out tiles (atomicAdd); the CTA that completes a phase's last tile
// applies the stopping rule where the phase has one and publishes the next phase (atomicExch), so
// grids advance independently and the small levels of one grid run beside the large levels of
// another.  A CTA only waits for phases whose tiles running CTAs hold: nothing depends on every CTA
// being resident.  Every wait is bounded (globaltimer); a CTA that gives up raises the error flag of
// every unfinished grid and the batch's own flag, and the other CTAs leave when they see it.
// The per-cell arithmetic is that of the quad kernels, so a grid's iterate is the one its own
// launch-by-launch solve produces, up to the order of the FP64 norm and mean reductions.
enum { PP_INIT = 0, PP_DEFECT, PP_SWEEP0, PP_SWEEP, PP_SWEEP_ACC, PP_RESTRICT, PP_PROLONG, PP_COARSE, PP_CONVERT };
enum { PT_NONE = 0, PT_START = 1, PT_STEP = 2 };

struct PPhase {
    int type, level, zc, gx;
    int nvb, per, ntiles, test;  // 256-thread blocks, blocks per tile (a multiple of 4), tiles, stopping rule
    int cnx, cny, cnz, pack;     // coarse level extents (restriction, prolongation); coarse pack index
    float* dst;
    const float* src;
    const float* f;
};

struct PGrid {
    Lvl<float> L[kMaxLevels];
    Lvl<double> L0;        // FP64 view of the finest level
    const PPhase* ph;
    const LPack* packs;
    MgLoop* loop;          // the handle's loop state (cycles, steps, relative residual history)
    double* acc;           // the handle's slots: ||r||^2, ||f||^2, sum of f over active cells, their count
    int* err;              // the handle's device error flag
    double* p64;
    float* r32;
    const float* f;        // finest right-hand side
    float* dst;            // FP32 copy of the solution
    int nph, loop_pc, end_pc, nu1, nu2, citers, prolong;
    float w;
};

struct __align__(64) PState {
    unsigned long long word;  // [63:48] phase, [47:32] its tiles, [31:0] next tile to hand out
    int done;                 // tiles of the current phase completed
    int finished;             // the grid's program has ended
};

struct PCtl {
    int withhold;             // test only: >= 0, the completion of this phase of the first grid is not published
    int prof;                 // 1: thread 0 of every CTA adds its cycles per activity to PArgs::prof
    unsigned long long lim;   // wait limit, ns
};
// PArgs::prof slots: waiting for work, tiles taken, descriptor setup, completion/publication, then per
// phase type its tile cycles and tiles
constexpr int kProfSlots = 4 + 2 * 9;

struct PArgs {
    const PGrid* grids;       // costliest first: the order the CTAs look for work in
    PState* st;
    unsigned* fin;            // grids whose program has ended
    int* err;                 // a CTA gave up waiting: the others leave too
    const PCtl* ctl;
    unsigned long long* prof;
    int count;
};

__host__ __device__ inline unsigned long long pp_word(int pc, int ntiles, unsigned next) {
    return ((unsigned long long)(unsigned)pc << 48) | ((unsigned long long)(unsigned)ntiles << 32) | next;
}

__global__ void pb_init_kernel(PArgs A, int max_cycles, int use_tol, double tol, int inner) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g == 0) {
        *A.fin = 0u;
        *A.err = 0;
    }
    if (g >= A.count) return;
    const PGrid& G = A.grids[g];
    for (int k = 0; k < 4; ++k) G.acc[k] = 0.0;
    MgLoop* st = G.loop;
    st->cycles = 0;
    st->steps = 0;
    st->max_cycles = max_cycles;
    st->use_tol = use_tol;
    st->inner = inner;
    st->tol = tol;
    st->rel = 0.0;
    A.st[g].word = pp_word(0, G.ph[0].ntiles, 0u);
    A.st[g].done = 0;
    A.st[g].finished = 0;
}

// One attempt at a tile of grid k (lane-private): true with (phase, tile) when one was free.
__device__ __forceinline__ bool pb_take(PState* S, int& pc, int& t) {
    const unsigned long long o = atomicAdd(&S->word, 1ull);
    if ((unsigned)(o & 0xffffffffu) >= (unsigned)((o >> 32) & 0xffffu)) return false;
    pc = (int)(o >> 48);
    t = (int)(o & 0xffffffffu);
    return true;
}

// A tile of some grid's current phase, looked for by the 32 lanes of warp 0 together: first the grid
// the CTA worked on last (pref), then every grid's word loaded at once, one per lane, and the first
// grid (in the costliest-first order) with a free tile taken.  Returns the grid or -1.
__device__ __forceinline__ int pb_grab(const PArgs& A, int pref, int& pc, int& t) {
    const int lane = threadIdx.x & 31;
    int got = 0;
    if (pref >= 0) {
        if (lane == 0) got = pb_take(A.st + pref, pc, t) ? 1 : 0;
        if (__shfl_sync(0xffffffffu, got, 0)) {
            pc = __shfl_sync(0xffffffffu, pc, 0);
            t = __shfl_sync(0xffffffffu, t, 0);
            return pref;
        }
    }
    for (int base = 0; base < A.count; base += 32) {
        const int k = base + lane;
        bool free = false;
        if (k < A.count) {
            const unsigned long long w = *reinterpret_cast<volatile unsigned long long*>(&A.st[k].word);
            free = (unsigned)(w & 0xffffffffu) < (unsigned)((w >> 32) & 0xffffu);
        }
        for (unsigned m = __ballot_sync(0xffffffffu, free); m; m &= m - 1) {
            const int lead = __ffs(m) - 1;
            if (lane == lead) got = pb_take(A.st + k, pc, t) ? 1 : 0;
            if (__shfl_sync(0xffffffffu, got, lead)) {
                pc = __shfl_sync(0xffffffffu, pc, lead);
                t = __shfl_sync(0xffffffffu, t, lead);
                return base + lead;
            }
        }
    }
    return -1;
}

// the stopping rule after a defect (mg_loop_start_kernel / mg_loop_check_kernel); true: one more step
__device__ bool pb_test(const PGrid& G, int test) {
    double nf2 = __ldcg(G.acc + 1);
    if (!(nf2 > 0.0)) nf2 = 1.0;
    const double rel = sqrt(__ldcg(G.acc) / nf2);
    volatile MgLoop* st = G.loop;
    st->rel = rel;
    if (test == PT_START) return !(st->use_tol && rel <= st->tol) && st->max_cycles > 0 && isfinite(rel);
    const int k = st->steps, c = st->cycles + st->inner;
    if (k < 64) st->hist[k] = rel;
    st->steps = k + 1;
    st->cycles = c;
    return !(st->use_tol && rel <= st->tol) && c < st->max_cycles && isfinite(rel);
}

// thread 0, after the CTA finished tile work of (g, pc)
__device__ void pb_complete(const PArgs& A, int g, int pc) {
    const PGrid& G = A.grids[g];
    PState* S = A.st + g;
    const PPhase& P = G.ph[pc];
    __threadfence();
    if (atomicAdd(&S->done, 1) + 1 != P.ntiles) return;
    atomicExch(&S->done, 0);
    if (g == 0 && pc == A.ctl->withhold) return;  // test only: the next phase is never published
    int npc = pc + 1;
    if (P.test != PT_NONE) npc = pb_test(G, P.test) ? G.loop_pc : G.end_pc;
    if (npc >= G.nph) {
        atomicExch(&S->finished, 1);
        __threadfence();
        atomicAdd(A.fin, 1u);
        return;
    }
    const PPhase& N = G.ph[npc];
    if (N.type == PP_DEFECT) atomicExch(reinterpret_cast<unsigned long long*>(G.acc), 0ull);
    __threadfence();
    atomicExch(&S->word, pp_word(npc, N.ntiles, 0u));
}

// a wait ran out: every grid still running reports it, and the other CTAs leave
__device__ void pb_give_up(const PArgs& A) {
    atomicOr(A.err, 2);
    for (int k = 0; k < A.count; ++k)
        if (*reinterpret_cast<volatile int*>(&A.st[k].finished) == 0) atomicOr(A.grids[k].err, 2);
}

// sum of v over the CTA's 32 warps, added to *out by thread 0
__device__ __forceinline__ void pb_cta_sum(double v, double* out, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < 32; ++k) t += red[k];
        atomicAdd(out, t);
    }
    __syncthreads();
}

// Loads of data written earlier in the launch.  Every tile starts after thread 0's GPU-scope fence
// that follows the atomic which handed the tile out (an acquire, ordered before the CTA's loads by
// the barrier after it), and every producer's stores precede a GPU-scope fence and the atomic that
// reports its tile done (a release): the memory model orders the tile's ordinary loads after the
// producers' stores, so they may go through L1 (false) instead of L2 only (true).
constexpr bool kPbCG = false;

// The work of one tile, one function per phase type (each with its own register allocation: the
// persistent kernel's 1024 threads leave 64 registers a thread).  vb0 .. v1 - 1: the tile's blocks.
__device__ __noinline__ void pb_sweep0(const PPhase& Ps, const Lvl<float>& Ls, float w, int vb0, int v1, int tid) {
    const PPhase P = Ps;
    const Lvl<float> L = Ls;
    for (int vb = vb0; vb < v1; vb += 4) jacobi0_q_body<float, kPbCG>(P.dst, P.f, L, w, P.zc, vb % P.gx, vb / P.gx, tid);
}
__device__ __noinline__ void pb_sweep(const PPhase& Ps, const Lvl<float>& Ls, float w, int vb0, int v1, int tid) {
    const PPhase P = Ps;
    const Lvl<float> L = Ls;
    for (int vb = vb0; vb < v1; vb += 4)
        jacobi_q_body<float, false, kPbCG>(P.dst, P.src, P.f, L, w, P.zc, nullptr, vb % P.gx, vb / P.gx, tid);
}
__device__ __noinline__ void pb_sweep_acc(const PPhase& Ps, const Lvl<float>& Ls, float w, double* p64, int vb0,
                                          int v1, int tid) {
    const PPhase P = Ps;
    const Lvl<float> L = Ls;
    for (int vb = vb0; vb < v1; vb += 4)
        jacobi_q_body<float, true, kPbCG>(nullptr, P.src, P.f, L, w, P.zc, p64, vb % P.gx, vb / P.gx, tid);
}
__device__ __noinline__ void pb_restrict(const PPhase& Ps, const Lvl<float>& Ls, int vb0, int v1, int tid) {
    const PPhase P = Ps;
    const Lvl<float> L = Ls;
    for (int vb = vb0; vb < v1; vb += 4)
        resid_restrict_q_body<float, kPbCG>(P.dst, P.src, P.f, L, P.cnx, P.cny, P.cnz, P.zc, vb % P.gx, vb / P.gx, tid);
}
__device__ __noinline__ void pb_prolong(const PPhase& Ps, const Lvl<float>& Ls, int vb0, int v1, int tid) {
    const PPhase P = Ps;
    const Lvl<float> L = Ls;
    for (int vb = vb0; vb < v1; vb += 4)
        prolong_tri_q_body<float, kPbCG>(P.dst, P.src, L.nx, L.ny, L.nz, P.cnx, P.cny, P.cnz, vb % P.gx, vb / P.gx, tid);
}
__device__ __noinline__ void pb_coarse(const LPack& Q, const PGrid& G, float* lean_smem) {
    lean_cycle<true>(Q, G.nu1, G.nu2, G.w, G.citers, G.prolong, lean_smem);
}
// active-cell sum and count of f (active_sum_q_kernel), ||f||^2 (sumsq_kernel), p64 = 0
__device__ __noinline__ void pb_init(const PPhase& Ps, const Lvl<double>& Ls, const float* f, double* p64, int vb0,
                                     int v1, int tid, double* out) {
    const PPhase P = Ps;
    const Lvl<double> L = Ls;
    double sf = 0.0, cnt = 0.0, sq = 0.0;
    const int nq = L.ny >> 2;
    for (int vb = vb0; vb < v1; vb += 4) {
        const long q = (long)(vb % P.gx) * 256 + tid;
        const int z0 = (vb / P.gx) * P.zc, z1 = min(z0 + P.zc, L.nz);
        if (q >= (long)L.nx * nq || z0 >= z1) continue;
        const int x = (int)(q / nq), y0 = (int)(q - (long)x * nq) * 4;
        QCol<double, float> col(L, f, x, y0, z0);
        for (int z = z0; z < z1; ++z) {
            const long i = col.i;
            Q4<double> dg, od, c;
            col.step(dg, od, c);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (dg.a[k] > kEps) { sf += c.a[k]; cnt += 1.0; }
                sq += c.a[k] * c.a[k];
            }
            st4(p64 + i, zero4<double>());
        }
    }
    out[0] = sf;
    out[1] = cnt;
    out[2] = sq;
}
__device__ __noinline__ double pb_defect(const PPhase& Ps, const Lvl<double>& Ls, const PGrid& G, double m, int vb0,
                                         int v1, int tid) {
    const PPhase P = Ps;
    const Lvl<double> L = Ls;
    float* const r32 = G.r32;
    const double* const p64 = G.p64;
    const float* const f = G.f;
    double s2 = 0.0;
    for (int vb = vb0; vb < v1; vb += 4)
        s2 += defect64_q_body<double, kPbCG>(r32, p64, f, L, m, P.zc, vb % P.gx, vb / P.gx, tid);
    return s2;
}

__global__ void __launch_bounds__(1024, 1) batch_persist_kernel(PArgs A) {
    extern __shared__ __align__(16) float lean_smem[];
    __shared__ Lvl<float> sL;
    __shared__ Lvl<double> sD;
    __shared__ PPhase sP;
    __shared__ double red[32];
    __shared__ int job[3];
    const int sub = threadIdx.x >> 8, tid = threadIdx.x & 255;
    int last = -1;  // the grid of the CTA's previous tile (warp 0)
    const bool prof = A.ctl->prof != 0;
    long long c0 = 0, c1 = 0, c2 = 0, c3 = 0;  // thread 0: cycle stamps of one tile's stages
    for (;;) {
        if (threadIdx.x < 32) {
            int g = -1, pc = 0, t = 0;
            if (prof && threadIdx.x == 0) c0 = clock64();
            const unsigned long long t0 = wptc::globaltimer();
            for (;;) {
                if (*reinterpret_cast<volatile int*>(A.err) != 0) break;
                if ((g = pb_grab(A, last, pc, t)) >= 0) break;
                if (*reinterpret_cast<volatile unsigned*>(A.fin) >= (unsigned)A.count) break;
                int out = 0;
                if (threadIdx.x == 0 && wptc::globaltimer() - t0 > A.ctl->lim) {
                    pb_give_up(A);
                    out = 1;
                }
                if (__shfl_sync(0xffffffffu, out, 0)) break;
                __nanosleep(128);
            }
            last = g;
            if (threadIdx.x == 0) {
                if (prof) {
                    c1 = clock64();
                    atomicAdd(A.prof + 0, (unsigned long long)(c1 - c0));
                    if (g >= 0) atomicAdd(A.prof + 1, 1ull);
                }
                job[0] = g;
                job[1] = pc;
                job[2] = t;
                __threadfence();
            }
        }
        __syncthreads();
        const int g = job[0];
        if (g < 0) return;
        const int pc = job[1], t = job[2];
        const PGrid& G = A.grids[g];
        {
            const PPhase* gp = G.ph + pc;
            constexpr int nP = sizeof(PPhase) / 4, nL = sizeof(Lvl<float>) / 4, nD = sizeof(Lvl<double>) / 4;
            static_assert(nP <= 64 && nL <= 64 && nD <= 64, "descriptor copy: one word per thread");
            const int lev = gp->level;
            if (threadIdx.x < nP)
                reinterpret_cast<unsigned*>(&sP)[threadIdx.x] = reinterpret_cast<const unsigned*>(gp)[threadIdx.x];
            else if (threadIdx.x >= 64 && threadIdx.x < 64 + nL)
                reinterpret_cast<unsigned*>(&sL)[threadIdx.x - 64] =
                    reinterpret_cast<const unsigned*>(&G.L[lev])[threadIdx.x - 64];
            else if (threadIdx.x >= 128 && threadIdx.x < 128 + nD)
                reinterpret_cast<unsigned*>(&sD)[threadIdx.x - 128] =
                    reinterpret_cast<const unsigned*>(&G.L0)[threadIdx.x - 128];
        }
        __syncthreads();
        if (prof && threadIdx.x == 0) c2 = clock64();
        const int type = sP.type;
        const int vb0 = sP.per * t + sub, v1 = min(sP.per * (t + 1), sP.nvb);
        switch (type) {
            case PP_COARSE: pb_coarse(G.packs[sP.pack], G, lean_smem); break;
            case PP_INIT: {
                double o[3];
                pb_init(sP, sD, G.f, G.p64, vb0, v1, tid, o);
                pb_cta_sum(o[0], G.acc + 2, red);
                pb_cta_sum(o[1], G.acc + 3, red);
                pb_cta_sum(o[2], G.acc + 1, red);
                break;
            }
            case PP_DEFECT: {
                const double m = __ldcg(G.acc + 2) / fmax(__ldcg(G.acc + 3), 1.0);
                pb_cta_sum(pb_defect(sP, sD, G, m, vb0, v1, tid), G.acc, red);
                break;
            }
            case PP_CONVERT: {
                const long n = (long)sL.nx * sL.ny * sL.nz;
                for (int vb = vb0; vb < v1; vb += 4) {
                    const long i = (long)vb * 1024 + 4L * tid;
                    if (i < n) st4(G.dst + i, cvt4<float>(ldq<kPbCG>(G.p64 + i)));
                }
                break;
            }
            case PP_SWEEP0: pb_sweep0(sP, sL, G.w, vb0, v1, tid); break;
            case PP_SWEEP: pb_sweep(sP, sL, G.w, vb0, v1, tid); break;
            case PP_SWEEP_ACC: pb_sweep_acc(sP, sL, G.w, G.p64, vb0, v1, tid); break;
            case PP_RESTRICT: pb_restrict(sP, sL, vb0, v1, tid); break;
            default: pb_prolong(sP, sL, vb0, v1, tid); break;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            if (prof) c3 = clock64();
            pb_complete(A, g, pc);
            if (prof) {
                atomicAdd(A.prof + 2, (unsigned long long)(c2 - c1));
                atomicAdd(A.prof + 3, (unsigned long long)(clock64() - c3));
                atomicAdd(A.prof + 4 + 2 * type, (unsigned long long)(c3 - c2));
                atomicAdd(A.prof + 5 + 2 * type, 1ull);
            }
        }
    }
}

// The tiles of a phase: nvb blocks of cells_vb cells, about `target` cells per tile (a multiple of
// four blocks, one per sub-block), at least one tile, at most 65535.
void pp_tiles(PPhase& q, long nvb, long cells_vb, long target) {
    long per = (target + cells_vb - 1) / cells_vb;
    per = std::max(4L, (per + 3) / 4 * 4);
    long nt = (nvb + per - 1) / per;
    while (nt > 65535) {
        per *= 2;
        nt = (nvb + per - 1) / per;
    }
    q.nvb = (int)nvb;
    q.per = (int)per;
    q.ntiles = (int)std::max(1L, nt);
}

// One grid's program (PGrid's phases and coarse packs), built by mirroring the buffer swaps of the
// launch-by-launch cycle on copies of the level pointers (the handle is not changed).
struct PBuild {
    wp_mgfrac3d* h;
    int nu1, nu2, lc;
    long target;
    float* v[kMaxLevels];
    float* t[kMaxLevels];
    std::vector<PPhase> ph;
    std::vector<LPack> packs;

    PPhase base(int type, int l) const {
        PPhase q;
        memset(&q, 0, sizeof(q));
        q.type = type;
        q.level = l;
        return q;
    }
    static int zc_of(const Level& L) { return std::max(1, std::min(L.n[2], 8)); }
    static long quads(const Level& L) { return (long)wp_cdiv((size_t)L.n[0] * (L.n[1] / 4), 256); }
    // a finest-level column phase (INIT, DEFECT) on the quad tiling
    void column(int type, int test) {
        const Level& L = h->lv[0];
        PPhase q = base(type, 0);
        q.zc = zc_of(L);
        q.gx = (int)quads(L);
        q.test = test;
        pp_tiles(q, q.gx * (long)wp_cdiv(L.n[2], q.zc), 1024L * q.zc, target);
        ph.push_back(q);
    }
    void cycle(int l, const float* f, bool clear, bool acc) {
        if (l == lc) {
            LPack Q;
            memset(&Q, 0, sizeof(Q));
            Q.n = h->nl - lc;
            for (int k = 0; k < Q.n; ++k) {
                Level& E = h->lv[lc + k];
                Q.lv[k] = {E.n[0], E.n[1], E.n[2], E.ccf, v[lc + k], t[lc + k], E.f};
            }
            PPhase q = base(PP_COARSE, l);
            q.pack = (int)packs.size();
            q.nvb = q.per = q.ntiles = 1;
            packs.push_back(Q);
            ph.push_back(q);
            for (int k = 0; k < Q.n; ++k) {
                const int swaps = (k == Q.n - 1) ? h->coarsest_iters : nu1 + nu2;
                if (swaps & 1) std::swap(v[lc + k], t[lc + k]);
            }
            return;
        }
        const Level& L = h->lv[l];
        const Level& C = h->lv[l + 1];
        const int zc = zc_of(L);
        const long gx = quads(L);
        auto sweep = [&](int type) {
            PPhase q = base(type, l);
            q.zc = zc;
            q.gx = (int)gx;
            q.dst = type == PP_SWEEP_ACC ? nullptr : t[l];
            q.src = v[l];
            q.f = f;
            pp_tiles(q, gx * (long)wp_cdiv(L.n[2], zc), 1024L * zc, target);
            ph.push_back(q);
            std::swap(v[l], t[l]);
        };
        int pre = nu1;
        if (clear) {
            sweep(PP_SWEEP0);
            pre = nu1 - 1;
        }
        for (int k = 0; k < pre; ++k) sweep(PP_SWEEP);
        {
            const int czc = std::max(1, zc / 2);
            PPhase q = base(PP_RESTRICT, l);
            q.zc = czc;
            q.gx = (int)wp_cdiv((size_t)C.n[0] * (L.n[1] / 4) * 2, 256);
            q.dst = C.f;
            q.src = v[l];
            q.f = f;
            q.cnx = C.n[0];
            q.cny = C.n[1];
            q.cnz = C.n[2];
            pp_tiles(q, q.gx * (long)wp_cdiv(C.n[2], czc), 2048L * czc, target);
            ph.push_back(q);
        }
        cycle(l + 1, C.f, true, false);
        {
            PPhase q = base(PP_PROLONG, l);
            q.gx = (int)gx;
            q.dst = v[l];
            q.src = v[l + 1];
            q.cnx = C.n[0];
            q.cny = C.n[1];
            q.cnz = C.n[2];
            pp_tiles(q, gx * (long)L.n[2], 1024L, target);
            ph.push_back(q);
        }
        for (int k = 0; k < nu2; ++k) sweep(acc && k == nu2 - 1 ? PP_SWEEP_ACC : PP_SWEEP);
    }
};

// Whether handle h can run its mixed solve as a persistent program (quad levels with aligned work
// arrays down to a lean coarse pack that fits the CTA's shared memory): the pack's first level, its
// shared bytes, or -1 with a message.
int persist_plan(wp_mgfrac3d* h, const wp_mg_params* prm, size_t smem_cap, size_t* lean_bytes, const char** why) {
    *why = nullptr;
    if (prm->prolongation != WP_PROLONG_TRILINEAR || prm->nu1 < 1 || prm->nu2 < 1 || prm->start == WP_START_FMG) {
        *why = "the persistent batch runs trilinear V(nu1, nu2) cycles with nu1, nu2 >= 1 from a zero start";
        return -1;
    }
    if (!h->p64 || !h->r32 || !h->loop_state) {
        *why = "mixed-precision work arrays not prepared";
        return -1;
    }
    int lc = -1;
    for (int l = 1; l < h->nl - 1 && lc < 0; ++l) {
        long pack = 0;
        for (int k = l; k < h->nl; ++k) pack += h->lv[k].cells;
        if (h->lv[l].cells <= kCoarseCells && h->nl - l <= kCoarseMax && pack <= kCoarseSmemCells) lc = l;
    }
    if (lc < 1) {
        *why = "a grid has no coarse level of at most 4096 cells for the single-CTA coarse cycle";
        return -1;
    }
    for (int l = 0; l < lc; ++l) {
        const Level& L = h->lv[l];
        const Level& C = h->lv[l + 1];
        if (!quad_ok(L) || C.n[1] * 2 != L.n[1] || !al16(L.v) || !al16(L.t) || (l > 0 && !al16(L.f)) ||
            !al16(h->r32) || !al16(h->p64)) {
            *why = "a level above the coarse pack has a y extent that is not a multiple of 4 (or is not halved)";
            return -1;
        }
    }
    LPack Q;
    Q.n = h->nl - lc;
    for (int k = 0; k < Q.n; ++k) {
        const Level& E = h->lv[lc + k];
        if (!E.ccf) {
            *why = "a coarse level has no precomputed stencils";
            return -1;
        }
        Q.lv[k] = {E.n[0], E.n[1], E.n[2], E.ccf, E.v, E.t, E.f};
    }
    *lean_bytes = sizeof(float) * (size_t)lean_smem_floats(Q, true);
    if (*lean_bytes > smem_cap) {
        *why = "a grid's coarse pack does not fit the persistent CTA's shared memory";
        return -1;
    }
    return lc;
}

// Builds handle h's program into ph / packs and fills its descriptor (device pointers of the
// program arrays are set by the caller).
void persist_program(wp_mgfrac3d* h, const wp_mg_params* prm, float* dst, const float* f, long target, int lc,
                     PGrid* G, std::vector<PPhase>& ph, std::vector<LPack>& packs) {
    PBuild b;
    b.h = h;
    b.nu1 = prm->nu1;
    b.nu2 = prm->nu2;
    b.lc = lc;
    b.target = target;
    for (int l = 0; l < h->nl; ++l) {
        b.v[l] = h->lv[l].v;
        b.t[l] = h->lv[l].t;
    }
    b.column(PP_INIT, PT_NONE);
    b.column(PP_DEFECT, PT_START);
    const int loop_pc = (int)b.ph.size();
    const int inner = inner_of(prm);
    for (int j = 0; j < inner; ++j) b.cycle(0, h->r32, j == 0, j == inner - 1);
    b.column(PP_DEFECT, PT_STEP);
    const int end_pc = (int)b.ph.size();
    {
        PPhase q = b.base(PP_CONVERT, 0);
        pp_tiles(q, (long)wp_cdiv(h->lv[0].cells, 1024), 1024L, target);
        b.ph.push_back(q);
    }
    memset(G, 0, sizeof(*G));
    for (int l = 0; l <= lc; ++l) G->L[l] = view<float>(h->lv[l]);
    G->L0 = view<double>(h->lv[0]);
    G->loop = reinterpret_cast<MgLoop*>(h->loop_state);
    G->acc = h->acc;
    G->err = reinterpret_cast<int*>(h->acc + 4);
    G->p64 = h->p64;
    G->r32 = h->r32;
    G->f = f;
    G->dst = dst;
    G->nph = (int)b.ph.size();
    G->loop_pc = loop_pc;
    G->end_pc = end_pc;
    G->nu1 = prm->nu1;
    G->nu2 = prm->nu2;
    G->citers = h->coarsest_iters;
    G->prolong = prm->prolongation;
    G->w = (float)prm->omega;
    ph.swap(b.ph);
    packs.swap(b.packs);
}

}  // namespace

// Many handles' mixed solves as one persistent launch (see batch_persist_kernel).
struct wp_mg_pbatch {
    int count = 0;
    PGrid* d_grids = nullptr;
    PState* d_st = nullptr;
    unsigned* d_fin = nullptr;  // then the batch's error flag (the int after it)
    PCtl* d_ctl = nullptr;
    PCtl ctl{-1, 0, 0};         // the control block's value on the device
    unsigned long long* d_prof = nullptr;  // kProfSlots counters (see PCtl::prof)
    std::vector<void*> blobs;   // per grid: phases, then coarse packs
    size_t smem = 0;
    int grid = 0;
    wp_mg_params prm;
    long target = 0;
    long long tiles = 0;        // tiles of one pass of every grid's program (report)
};

namespace {

void pbatch_free(wp_mg_pbatch* pb) {
    for (void* p : pb->blobs) cudaFree(p);
    if (pb->d_grids) cudaFree(pb->d_grids);
    if (pb->d_st) cudaFree(pb->d_st);
    if (pb->d_fin) cudaFree(pb->d_fin);
    if (pb->d_ctl) cudaFree(pb->d_ctl);
    if (pb->d_prof) cudaFree(pb->d_prof);
    delete pb;
}

}  // namespace

// Builds the persistent program of every handle (hs[i] solves f[i] into dst[i] and its FP64 iterate;
// the mixed work arrays prepared).  The CTAs look for work in the order given.  target_cells:
// cells per tile (0 = 32768).  WP_ERR_UNSUPPORTED when a handle's levels do not fit the program.
wp_status wp_mg_pbatch_create(wp_mg_pbatch** out, wp_mgfrac3d* const* hs, float* const* dst, const float* const* f,
                              int count, const wp_mg_params* prm, long target_cells) {
    *out = nullptr;
    if (count < 1 || !hs || !dst || !f || !prm) {
        wp_set_error_msg("persistent batch: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    cudaFuncAttributes fa;
    WP_CUDA_TRY(cudaFuncGetAttributes(&fa, batch_persist_kernel));
    int dev = 0, optin = 0;
    WP_CUDA_TRY(cudaGetDevice(&dev));
    WP_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t cap = (size_t)optin > fa.sharedSizeBytes + 1024 ? (size_t)optin - fa.sharedSizeBytes - 1024 : 0;
    wp_mg_pbatch* pb = new (std::nothrow) wp_mg_pbatch();
    if (!pb) return WP_ERR_INVALID_ARG;
    pb->count = count;
    pb->prm = *prm;
    pb->target = target_cells > 0 ? target_cells : 32768;
    std::vector<PGrid> G(count);
    wp_status st = WP_OK;
    for (int i = 0; i < count && st == WP_OK; ++i) {
        size_t lean = 0;
        const char* why = nullptr;
        const int lc = persist_plan(hs[i], prm, cap, &lean, &why);
        if (lc < 0) {
            wp_set_error_msg(why);
            st = WP_ERR_UNSUPPORTED;
            break;
        }
        pb->smem = std::max(pb->smem, lean);
        std::vector<PPhase> ph;
        std::vector<LPack> packs;
        persist_program(hs[i], prm, dst[i], f[i], pb->target, lc, &G[i], ph, packs);
        hs[i]->last64 = 1;  // the FP64 iterate of the last solve is p64
        for (const PPhase& q : ph) pb->tiles += q.ntiles;
        const size_t bph = sizeof(PPhase) * ph.size(), bpk = sizeof(LPack) * packs.size();
        const size_t off = (bph + 255) / 256 * 256;
        void* blob = nullptr;
        cudaError_t e = cudaMalloc(&blob, off + bpk + 16);
        if (e == cudaSuccess) {
            pb->blobs.push_back(blob);
            e = cudaMemcpy(blob, ph.data(), bph, cudaMemcpyHostToDevice);
        }
        if (e == cudaSuccess && bpk) e = cudaMemcpy((char*)blob + off, packs.data(), bpk, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            wp_set_cuda_error(e, "persistent batch programs", __FILE__, __LINE__);
            st = WP_ERR_CUDA;
            break;
        }
        G[i].ph = reinterpret_cast<const PPhase*>(blob);
        G[i].packs = reinterpret_cast<const LPack*>((char*)blob + off);
    }
    if (st == WP_OK) {
        cudaError_t e = cudaMalloc((void**)&pb->d_grids, sizeof(PGrid) * count);
        if (e == cudaSuccess) e = cudaMalloc((void**)&pb->d_st, sizeof(PState) * count);
        if (e == cudaSuccess) e = cudaMalloc((void**)&pb->d_fin, 2 * sizeof(unsigned));
        if (e == cudaSuccess) e = cudaMalloc((void**)&pb->d_ctl, sizeof(PCtl));
        if (e == cudaSuccess) e = cudaMalloc((void**)&pb->d_prof, sizeof(unsigned long long) * kProfSlots);
        if (e == cudaSuccess) e = cudaMemset(pb->d_prof, 0, sizeof(unsigned long long) * kProfSlots);
        if (e == cudaSuccess) e = cudaMemcpy(pb->d_grids, G.data(), sizeof(PGrid) * count, cudaMemcpyHostToDevice);
        pb->ctl.withhold = -1;
        pb->ctl.lim = wptc::kWaitLimitNs;
        if (e == cudaSuccess) e = cudaMemcpy(pb->d_ctl, &pb->ctl, sizeof(PCtl), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(batch_persist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)pb->smem);
        int per_sm = 0;
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_persist_kernel, 1024, pb->smem);
        if (e != cudaSuccess) {
            wp_set_cuda_error(e, "persistent batch setup", __FILE__, __LINE__);
            st = WP_ERR_CUDA;
        } else if (per_sm < 1) {
            wp_set_error_msg("persistent batch: a 1024-thread CTA with the coarse pack's shared memory does not fit an SM");
            st = WP_ERR_UNSUPPORTED;
        }
        pb->grid = wp_sm_count();
    }
    if (st != WP_OK) {
        pbatch_free(pb);
        return st;
    }
    *out = pb;
    return WP_OK;
}

// Test only: the next launches withhold the publication that follows phase `at` of the first grid
// (at < 0: none), and every wait of the launch gives up after limit_ns.  Enqueued on s.
wp_status wp_mg_pbatch_arm(wp_mg_pbatch* pb, int at, unsigned long long limit_ns, cudaStream_t s) {
    const PCtl c{at, pb->ctl.prof, limit_ns ? limit_ns : wptc::kWaitLimitNs};
    if (c.withhold == pb->ctl.withhold && c.lim == pb->ctl.lim) return WP_OK;
    pb->ctl = c;
    WP_CUDA_TRY(cudaMemcpyAsync(pb->d_ctl, &pb->ctl, sizeof(PCtl), cudaMemcpyHostToDevice, s));
    WP_CUDA_TRY(cudaStreamSynchronize(s));
    return WP_OK;
}

// The persistent kernel's activity counters: enable 1 clears them and switches the counting on for
// the following launches, 0 switches it off; out (may be NULL) receives the kProfSlots sums so far.
wp_status wp_mg_pbatch_profile(wp_mg_pbatch* pb, int enable, unsigned long long* out, cudaStream_t s) {
    WP_CUDA_TRY(cudaStreamSynchronize(s));
    if (out) WP_CUDA_TRY(cudaMemcpy(out, pb->d_prof, sizeof(unsigned long long) * kProfSlots, cudaMemcpyDeviceToHost));
    if (enable) WP_CUDA_TRY(cudaMemset(pb->d_prof, 0, sizeof(unsigned long long) * kProfSlots));
    if ((enable != 0) != (pb->ctl.prof != 0)) {
        pb->ctl.prof = enable != 0;
        WP_CUDA_TRY(cudaMemcpy(pb->d_ctl, &pb->ctl, sizeof(PCtl), cudaMemcpyHostToDevice));
    }
    return WP_OK;
}
int wp_mg_pbatch_prof_slots() { return kProfSlots; }

// The loop state and slots initialised, then the persistent kernel (two launches, capturable).
wp_status wp_mg_pbatch_launch(wp_mg_pbatch* pb, cudaStream_t s) {
    PArgs A;
    A.grids = pb->d_grids;
    A.st = pb->d_st;
    A.fin = pb->d_fin;
    A.err = reinterpret_cast<int*>(pb->d_fin + 1);
    A.ctl = pb->d_ctl;
    A.prof = pb->d_prof;
    A.count = pb->count;
    const wp_mg_params& p = pb->prm;
    WP_KERNEL("batch_persist_init", 0.0, s,
              pb_init_kernel<<<wp_cdiv(pb->count, 128), 128, 0, s>>>(A, p.max_cycles, p.rel_tol > 0.0 ? 1 : 0, p.rel_tol,
                                                                     inner_of(&p)));
    WP_KERNEL("batch_persistent", 0.0, s, batch_persist_kernel<<<pb->grid, 1024, pb->smem, s>>>(A));
    return WP_OK;
}

long long wp_mg_pbatch_tiles(const wp_mg_pbatch* pb) { return pb->tiles; }
size_t wp_mg_pbatch_smem(const wp_mg_pbatch* pb) { return pb->smem; }

void wp_mg_pbatch_destroy(wp_mg_pbatch* pb) {
    if (pb) pbatch_free(pb);
}

namespace {

wp_status residual_rel(wp_mgfrac3d* h, const float* v, const float* f, double* rel, cudaStream_t s) {
    if (!h || !v || !f || !rel) { wp_set_error_msg("wp_mgfrac_residual: null pointer"); return WP_ERR_INVALID_ARG; }
    double nr2 = 0.0, nf2 = 0.0;
    wp_status st = defect<float>(h, v, f, 0.0, nullptr, &nr2, &nf2, s);
    if (st != WP_OK) return st;
    *rel = std::sqrt(nr2) / std::sqrt(nf2);
    return WP_OK;
}

}  // namespace

extern "C" CUWHHD_API wp_status wp_mgfrac3d_create(wp_mgfrac3d** h, const float* ax, const float* ay, const float* az,
                                                   int nx, int ny, int nz, double dx, double dy, double dz, char bc,
                                                   void* stream) {
    return create_common(h, 3, ax, ay, az, nx, ny, nz, dx, dy, dz, bc, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_mgfrac3d_solve(wp_mgfrac3d* h, float* dst, const float* pre_v, const float* f,
                                                  int n_iters, int nu1, int nu2, double weight, void* stream) {
    return solve_fixed(h, dst, pre_v, f, n_iters, nu1, nu2, weight, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_mgfrac3d_solve_index(wp_mgfrac3d* h, float* dst, const float* pre_v,
                                                        const float* f, int n_iters, int nu1, int nu2, double weight,
                                                        void* stream) {
    return solve_index<float>(h, dst, pre_v, f, n_iters, nu1, nu2, weight, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_mgfrac3d_solve_index64(wp_mgfrac3d* h, double* dst, const double* pre_v,
                                                          const double* f, int n_iters, int nu1, int nu2,
                                                          double weight, void* stream) {
    return solve_index<double>(h, dst, pre_v, f, n_iters, nu1, nu2, weight, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_mgfrac3d_index_sizes(wp_mgfrac3d* h, long long* cells, long long* segments, int cap,
                                                        int* levels, void* stream) {
    if (!h || cap < 0) { wp_set_error_msg("wp_mgfrac3d_index_sizes: bad arguments"); return WP_ERR_INVALID_ARG; }
    if (h->dims != 3) { wp_set_error_msg("wp_mgfrac3d_index_sizes: the index-sparse cycle is 3D only"); return WP_ERR_UNSUPPORTED; }
    wp_status st = build_index(h, (cudaStream_t)stream);
    if (st != WP_OK) return st;
    if (levels) *levels = h->nl;
    for (int l = 0; l < h->nl && l < cap; ++l) {
        if (cells) cells[l] = h->lv[l].icells;
        if (segments) segments[l] = h->lv[l].iseg_n;
    }
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_mgfrac3d_solve_tol(wp_mgfrac3d* h, float* dst, const float* pre_v, const float* f,
                                                      const wp_mg_params* params, wp_mg_report* report, void* stream) {
    return solve_tol(h, dst, pre_v, f, params, report, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_mgfrac3d_residual(wp_mgfrac3d* h, const float* v, const float* f, double* rel,
                                                     void* stream) {
    return residual_rel(h, v, f, rel, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_mgfrac3d_iterate64(wp_mgfrac3d* h, double* dst, void* stream) {
    if (!h || !dst || h->last64 == 0) { wp_set_error_msg("wp_mgfrac3d_iterate64: no FP64 iterate available"); return WP_ERR_INVALID_ARG; }
    const double* src = h->last64 == 1 ? h->p64 : h->lv[0].v64;
    WP_CUDA_TRY(cudaMemcpyAsync(dst, src, sizeof(double) * h->lv[0].cells, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_mgfrac3d_iterate64_view(wp_mgfrac3d* h, const double** out) {
    if (!h || !out || h->last64 == 0) {
        wp_set_error_msg("wp_mgfrac3d_iterate64_view: no FP64 iterate available");
        return WP_ERR_INVALID_ARG;
    }
    *out = h->last64 == 1 ? h->p64 : h->lv[0].v64;
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_mgfrac3d_destroy(wp_mgfrac3d* h) {
    if (!h) return WP_OK;
    destroy_loop_graph(h);
    if (h->loop_state) cudaFree(h->loop_state);
    if (h->loop_cap) cudaStreamDestroy(h->loop_cap);
    destroy_levels(h);
    delete h;
    return WP_OK;
}

// 2D shares the implementation: a single z layer with no z faces
struct wp_mgfrac2d {
    wp_mgfrac3d* impl;
};

extern "C" CUWHHD_API wp_status wp_mgfrac2d_create(wp_mgfrac2d** h, const float* ax, const float* ay, int nx, int ny,
                                                   double dx, double dy, char bc, void* stream) {
    if (!h) { wp_set_error_msg("wp_mgfrac2d_create: null handle"); return WP_ERR_INVALID_ARG; }
    *h = nullptr;
    wp_mgfrac3d* impl = nullptr;
    wp_status st = create_common(&impl, 2, ax, ay, nullptr, nx, ny, 1, dx, dy, 1.0, bc, (cudaStream_t)stream);
    if (st != WP_OK) return st;
    wp_mgfrac2d* o = new (std::nothrow) wp_mgfrac2d();
    if (!o) { wp_mgfrac3d_destroy(impl); return WP_ERR_INVALID_ARG; }
    o->impl = impl;
    *h = o;
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_mgfrac2d_solve(wp_mgfrac2d* h, float* dst, const float* pre_v, const float* f,
                                                  int n_iters, int nu1, int nu2, double weight, void* stream) {
    if (!h) return WP_ERR_INVALID_ARG;
    return solve_fixed(h->impl, dst, pre_v, f, n_iters, nu1, nu2, weight, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_mgfrac2d_solve_tol(wp_mgfrac2d* h, float* dst, const float* pre_v, const float* f,
                                                      const wp_mg_params* params, wp_mg_report* report, void* stream) {
    if (!h) return WP_ERR_INVALID_ARG;
    return solve_tol(h->impl, dst, pre_v, f, params, report, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_mgfrac2d_residual(wp_mgfrac2d* h, const float* v, const float* f, double* rel,
                                                     void* stream) {
    if (!h) return WP_ERR_INVALID_ARG;
    return residual_rel(h->impl, v, f, rel, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_mgfrac2d_destroy(wp_mgfrac2d* h) {
    if (!h) return WP_OK;
    wp_mgfrac3d_destroy(h->impl);
    delete h;
    return WP_OK;
}

// ---- internal hooks used by the batched path (wp_batch.cu)
// ------------------------------------------------------------------ tile-shape autotuner
// Per level, times the column kernels (FP32 Jacobi sweep, fused residual-restriction, FP64 defect)
// over candidate z-chunks with CUDA events and keeps the fastest.  Results do not depend on the
// chunk (each cell's arithmetic is the same; only the grid shape changes).  Timings are cached per
// (device, kernel, extents) for the process, so later handles of the same shapes skip the search.
namespace {

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, int> g_tune_cache;

// reads the flush buffer (after it was written): the L2 then holds clean lines of it only, so the
// timed launch neither hits its own data nor pays for writing back someone else's
__global__ void flush_read_kernel(const uint4* __restrict__ p, size_t n, unsigned* __restrict__ sink) {
    unsigned acc = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        acc ^= p[i].x ^ p[i].w;
    if (acc == 0x9e3779b9u) sink[0] = acc;  // keeps the loads; practically never taken
}

// median of `reps` single launches, each timed alone; with a flush buffer the L2 is overwritten
// before every timed launch (a level larger than the L2 meets a cold cache inside a V-cycle)
template <typename F>
float time_launches(F&& launch, cudaStream_t s, cudaEvent_t a, cudaEvent_t b, int reps, void* flush,
                    size_t flush_bytes) {
    launch();
    std::vector<float> t;
    for (int r = 0; r < reps; ++r) {
        if (flush) {
            cudaMemsetAsync(flush, r & 0xff, flush_bytes, s);
            flush_read_kernel<<<wp_sm_count() * 4, 256, 0, s>>>(static_cast<const uint4*>(flush), flush_bytes / 16,
                                                                static_cast<unsigned*>(flush));
        }
        cudaEventRecord(a, s);
        launch();
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        t.push_back(ms);
    }
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

// CTAs of a column kernel for a z-chunk (to keep candidates that fill the GPU)
long grid_blocks(const Level& L, const Level* C, int kind, int zc) {
    const bool q = quad_ok(L) && (kind != kZcRestrict || (C && C->n[1] * 2 == L.n[1]));
    const int planes = kind == kZcRestrict ? C->n[2] : L.n[2];
    const long per_plane = q ? (long)wp_cdiv((size_t)(kind == kZcRestrict ? 2 * C->n[0] : L.n[0]) * (L.n[1] / 4), 256)
                             : (long)wp_cdiv(L.n[1], 32) * wp_cdiv(L.n[0], 8);
    return per_plane * wp_cdiv(planes, zc);
}

std::vector<int> zc_candidates(int nplanes) {
    std::vector<int> c;
    for (int z = 1; z <= nplanes; z *= 2) c.push_back(z);
    if (c.empty() || c.back() != nplanes) c.push_back(nplanes);
    return c;
}

wp_status autotune(wp_mgfrac3d* h, cudaStream_t s) {
    int dev = 0;
    WP_CUDA_TRY(cudaGetDevice(&dev));
    cudaEvent_t ea, eb;
    WP_CUDA_TRY(cudaEventCreate(&ea));
    WP_CUDA_TRY(cudaEventCreate(&eb));
    const bool prof = wp_profile_is_enabled();
    // the FP64 defect is tuned too (3D): its work arrays are those of the mixed solve
    if (h->dims == 3 && prepare_mixed(h) != WP_OK) return WP_ERR_CUDA;
    wp_profile_enable(0);
    const long long launches0 = wp_launch_count();
    wp_status st = WP_OK;
    // L2 flush buffer (twice the 126 MB L2), only if some level does not fit in the L2 by itself
    constexpr size_t kFlush = 256u << 20;
    constexpr long kL2Cells = (16L << 20) / 4;
    void* flush = nullptr;
    if (h->lv[0].cells > kL2Cells && cudaMalloc(&flush, kFlush) != cudaSuccess) {
        cudaGetLastError();
        flush = nullptr;
    }
    for (int l = 0; l < h->nl && st == WP_OK; ++l) {
        Level& L = h->lv[l];
        const int nx = L.n[0], ny = L.n[1], nz = L.n[2];
        if (nz == 1) { L.zc[0] = L.zc[1] = L.zc[2] = 1; continue; }
        // scratch contents: zero right-hand side and iterate (the level buffers are work arrays)
        cudaMemsetAsync(L.v, 0, sizeof(float) * L.cells, s);
        cudaMemsetAsync(L.f, 0, sizeof(float) * L.cells, s);
        const int kinds = (l == 0 && h->p64 && h->r32) ? 3 : (l + 1 < h->nl ? 2 : 1);
        for (int kind = 0; kind < kinds; ++kind) {
            const auto key = std::make_tuple(dev, kind, nx, ny, nz);
            {
                std::lock_guard<std::mutex> lk(g_tune_mu);
                auto it = g_tune_cache.find(key);
                if (it != g_tune_cache.end()) {
                    L.zc[kind] = it->second % 1000;
                    L.var[kind] = it->second / 1000;
                    continue;
                }
            }
            const Level* C = l + 1 < h->nl ? &h->lv[l + 1] : nullptr;
            const int planes = kind == kZcRestrict ? (C ? C->n[2] : 1) : nz;
            float best = 1e30f;
            int best_zc = level_zc(L, kind), best_var = 0;
            const long most = grid_blocks(L, C, kind, 1);
            const long floor_blocks = std::min<long>(most, 2L * wp_sm_count());
            void* fl = L.cells > kL2Cells ? flush : nullptr;
            // jacobi variants: 0-2 one sweep per launch (register budgets), 3 two sweeps per launch
            // jacobi 6 / restrict 4: one cell per thread (scalar column kernels), for levels small
            // enough that a quad per thread leaves too few threads
            const int nvar = !quad_ok(L) ? 1 : kind == kZcJacobi ? 7 : kind == kZcRestrict ? 5 : 2;
            for (int var = 0; var < nvar && st == WP_OK; ++var) {
                const bool two_sweeps = kind == kZcJacobi && var == 3;
                const bool staged = kind == kZcJacobi && var == 4;
                if (two_sweeps && !jacobi2_ok(L, L.f)) continue;
                if (staged && !jacobi_ts_ok(L, L.t, L.v, L.f)) continue;
                L.var[kind] = var;
                for (int zc : zc_candidates(planes)) {
                    // the TMA-staged sweep balances its own work over persistent CTAs: one timing
                    if (staged && zc != 1) continue;
                    long blocks = grid_blocks(L, C, kind, zc);
                    if (two_sweeps)
                        blocks = (long)((L.n[1] / 4 + J2_Q - 1) / J2_Q) * ((L.n[0] + J2_R - 1) / J2_R) *
                                 wp_cdiv(L.n[2], zc);
                    if ((kind == kZcJacobi && var == 6) || (kind == kZcRestrict && var == 4))
                        blocks = (long)wp_cdiv(L.n[1], 32) * wp_cdiv(L.n[0], 8) * wp_cdiv(planes, zc);
                    if (!staged && blocks < floor_blocks) continue;
                    auto launch = [&]() {
                        if (two_sweeps) launch_jacobi2<float>(L, L.t, L.v, L.f, 0.5f, zc, s);
                        else if (kind == kZcJacobi) launch_jacobi<float>(L, L.t, L.v, L.f, 0.5f, zc, s);
                        else if (kind == kZcRestrict) launch_resid_restrict<float>(L, *C, C->f, L.v, L.f, zc, s);
                        else launch_defect64<double>(L, h->r32, h->p64, L.f, 0.0, nullptr, h->acc, zc, s);
                    };
                    // the fused variant does two sweeps: compare time per sweep
                    const float ms = time_launches(launch, s, ea, eb, 5, fl, kFlush) / (two_sweeps ? 2.f : 1.f);
                    const cudaError_t e = cudaGetLastError();
                    if (e != cudaSuccess) { wp_set_cuda_error(e, "autotune", __FILE__, __LINE__); st = WP_ERR_CUDA; break; }
                    if (ms < best) { best = ms; best_zc = zc; best_var = var; }
                }
            }
            if (st != WP_OK) break;
            L.zc[kind] = best_zc;
            L.var[kind] = best_var;
            L.zc_ms[kind] = best;
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune_cache[key] = best_zc + 1000 * best_var;
        }
    }
    // the levels below the finest as one persistent launch, or launch by launch: time a V-cycle from
    // level 1 both ways (the levels are L2-resident: no flush) and keep the faster
    if (st == WP_OK && h->dims == 3 && h->nl >= 3 && !h->mid_forbid) {
        float best = 1e30f;
        int best_on = 1;
        for (int on = 1; on >= 0 && st == WP_OK; --on) {
            h->mid_on = on;
            Level& L1 = h->lv[1];
            auto launch = [&]() {
                vcycle<float>(h, 1, L1.f, 2, 2, 2.f / 3.f, WP_PROLONG_TRILINEAR, s, true);
            };
            const float ms = time_launches(launch, s, ea, eb, 5, nullptr, 0);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) { wp_set_cuda_error(e, "autotune", __FILE__, __LINE__); st = WP_ERR_CUDA; break; }
            if (ms < best) { best = ms; best_on = on; }
        }
        h->mid_on = best_on;
    }
    // level 0's V(2,2) cycle as the two fused passes or kernel by kernel: time both ways the pair of
    // cycles of one refinement step of the mixed solve (a cycle from zero, then one whose last sweep
    // adds into an FP64 iterate -- here a scratch array, not the handle's), after an L2 flush when
    // level 0 exceeds it; the fused passes only when they are clearly (5%) faster -- at 256^3 the
    // two measure alike and the one-sweep kernels use the memory bandwidth better per byte
    if (st == WP_OK && h->dims == 3 && h->nl >= 2 && h->lv[0].tuni) {
        Level& L0 = h->lv[0];
        double* acc = nullptr;
        if (cudaMalloc((void**)&acc, sizeof(double) * L0.cells) != cudaSuccess) {
            cudaGetLastError();
            acc = nullptr;
        }
        if (acc) {
            cudaMemsetAsync(acc, 0, sizeof(double) * L0.cells, s);
            float ms[2] = {0.f, 0.f};
            for (int on = 0; on < 2 && st == WP_OK; ++on) {
                h->fz_on = on;
                auto launch = [&]() {
                    vcycle<float>(h, 0, L0.f, 2, 2, 2.f / 3.f, WP_PROLONG_TRILINEAR, s, true);
                    bool added = false;
                    vcycle<float>(h, 0, L0.f, 2, 2, 2.f / 3.f, WP_PROLONG_TRILINEAR, s, false, acc, &added);
                };
                ms[on] = time_launches(launch, s, ea, eb, 5, flush, flush ? kFlush : 0);
                const cudaError_t e = cudaGetLastError();
                if (e != cudaSuccess) { wp_set_cuda_error(e, "autotune", __FILE__, __LINE__); st = WP_ERR_CUDA; break; }
            }
            cudaStreamSynchronize(s);
            cudaFree(acc);
            h->fz_on = ms[1] < 0.95f * ms[0] ? 1 : 0;
            ++h->tune_gen;
        }
    }
    if (flush) {
        cudaStreamSynchronize(s);
        cudaFree(flush);
    }
    wp_add_launches(-(wp_launch_count() - launches0));
    wp_profile_enable(prof ? 1 : 0);
    cudaEventDestroy(ea);
    cudaEventDestroy(eb);
    return st;
}

}  // namespace

extern "C" CUWHHD_API wp_status wp_mgfrac3d_autotune(wp_mgfrac3d* h, void* stream) {
    if (!h) { wp_set_error_msg("wp_mgfrac3d_autotune: null handle"); return WP_ERR_INVALID_ARG; }
    ++h->tune_gen;
    return autotune(h, (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_mgfrac3d_tiles(const wp_mgfrac3d* h, int* zc, int* variant, float* ms, int cap,
                                                   int* levels) {
    if (!h || (!zc && cap > 0)) { wp_set_error_msg("wp_mgfrac3d_tiles: null pointer"); return WP_ERR_INVALID_ARG; }
    if (levels) *levels = h->nl;
    for (int l = 0; l < h->nl; ++l)
        for (int k = 0; k < 3; ++k)
            if (3 * l + k < cap) {
                zc[3 * l + k] = level_zc(h->lv[l], k);
                if (variant) variant[3 * l + k] = h->lv[l].var[k];
                if (ms) ms[3 * l + k] = h->lv[l].zc_ms[k];
            }
    return WP_OK;
}

// Pins the chunk and kernel variant of one level's column kernel (kind 0 jacobi, 1 restrict,
// 2 defect); zc <= 0 restores the heuristic.
extern "C" CUWHHD_API wp_status wp_mgfrac3d_set_tile(wp_mgfrac3d* h, int level, int kind, int zc, int variant) {
    if (h && kind == 3 && (variant == 0 || variant == 1)) {
        // the levels below the finest: one persistent launch (1) or launch by launch (0)
        h->mid_on = variant;
        ++h->tune_gen;
        return WP_OK;
    }
    if (h && kind == 4 && (variant == 0 || variant == 1)) {
        // level 0's V(2,2) cycle: the two fused kernels (1) or one kernel per sweep / transfer (0)
        h->fz_on = variant;
        h->fz_zc = zc > 0 ? zc + (zc & 1) : 0;
        ++h->tune_gen;
        return WP_OK;
    }
    if (!h || level < 0 || level >= h->nl || kind < 0 || kind > 2 || variant < 0 || variant > 6 ||
        (kind == kZcRestrict && variant > 4) || (kind == kZcDefect && variant > 1)) {
        wp_set_error_msg("wp_mgfrac3d_set_tile: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    Level& L = h->lv[level];
    L.zc[kind] = zc > 0 ? zc : 0;
    L.var[kind] = variant;
    L.zc_ms[kind] = 0.f;
    ++h->tune_gen;
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_mgfrac3d_uniform_rows(const wp_mgfrac3d* h, int level, long long* uniform,
                                                         long long* rows) {
    if (!h || level < 0 || level >= h->nl || !uniform || !rows) {
        wp_set_error_msg("wp_mgfrac3d_uniform_rows: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    const Level& L = h->lv[level];
    *uniform = L.uni_rows;
    *rows = (long long)L.n[0] * L.n[2];
    return WP_OK;
}

wp_status wp_mg_prepare_mixed(wp_mgfrac3d* h) { return prepare_mixed(h); }
// a cooperative launch needs the whole GPU: the batch, whose grids run on concurrent graph branches,
// keeps every level launch by launch
void wp_mg_forbid_persistent(wp_mgfrac3d* h) { h->mid_forbid = 1; }
wp_status wp_mg_solve_mixed_loop_capture(wp_mgfrac3d* h, float* dst, const float* f, const wp_mg_params* prm,
                                         cudaStream_t s, long long* body_launches) {
    return solve_mixed_loop_capture(h, dst, f, prm, s, body_launches);
}
// the device loop's state (its first int is the V-cycle count of the last solve)
const void* wp_mg_loop_state(const wp_mgfrac3d* h) { return h->loop_state; }
wp_status wp_mg_solve_tol_internal(wp_mgfrac3d* h, float* dst, const float* f, const wp_mg_params* prm, wp_mg_report* r,
                                   cudaStream_t s) {
    return solve_tol(h, dst, nullptr, f, prm, r, s);
}
const double* wp_mg_slots(const wp_mgfrac3d* h) { return h->acc; }
// the FP64 iterate of the mixed solve (the batch's device loop leaves its result there)
const double* wp_mg_p64(const wp_mgfrac3d* h) { return h->p64; }
wp_mgfrac3d* wp_mg2d_impl(wp_mgfrac2d* h) { return h ? h->impl : nullptr; }
