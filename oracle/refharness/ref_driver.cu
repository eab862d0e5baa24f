// ref_driver.cu -- command-line driver around the reference's own CUDA classes.
//
// TEST INFRASTRUCTURE ONLY.  Linked against objects compiled from the unmodified reference
// sources (see Makefile in this directory); used on a GPU host to produce the golden fixtures in
// tests/golden/ and to time the reference build.  It calls only the reference's public entry
// points (CuWHHDForward::Solve1D, CuGetInnerProduct::GenerateIp, CuDivLocalProject3D,
// CuDivLocalProject, CuWaveletPotentialRecover3D/2D, CuMultigridFrac3D/2D, CuConvergence,
// CuGradient, CuSolidLevelSet3D, CuDst3D, CuParallelSweep3D) with the same call sequences as
// TestLocalProjection.cpp.
//
// Usage: ref_driver <op> <in_dir> <out_dir> [params...]; arrays are raw little-endian float64
// files <name>.bin in the reference layout (y fastest).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <chrono>

#include "cudaGlobal.cuh"
#include "cudaMath.cuh"
#include "WaveletTypes.h"
#include "cuWHHDForward.cuh"
#include "cuGetInnerProduct.cuh"
#include "cuDivLocalProject3D.cuh"
#include "cuDivLocalProject.cuh"
#include "cuWaveletPotentialRecover3D.cuh"
#include "cuWaveletPotentialRecover2D.cuh"
#include "cuMultigridFrac3D.cuh"
#include "cuMultigridFrac2D.cuh"
#include "cuWeightedJacobi3D.cuh"
#include "cuWeightedJacobi.cuh"
#include "cuConvergence.cuh"
#include "cuGradient.cuh"
#include "cuSolidLevelSet3D.cuh"
#include "cuFastSweeping.cuh"
#include "cuDst3D.cuh"
#include "cuParallelSweep3D.cuh"

static std::string g_in, g_out;

static std::vector<double> read_bin(const std::string& name, size_t n) {
    std::string path = g_in + "/" + name + ".bin";
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path.c_str()); exit(3); }
    std::vector<double> v(n);
    size_t got = fread(v.data(), sizeof(double), n, f);
    fclose(f);
    if (got != n) { fprintf(stderr, "short read %s: %zu of %zu\n", path.c_str(), got, n); exit(3); }
    return v;
}

static void write_bin(const std::string& name, const std::vector<double>& v) {
    std::string path = g_out + "/" + name + ".bin";
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(3); }
    fwrite(v.data(), sizeof(double), v.size(), f);
    fclose(f);
}

static DTYPE* to_dev(const std::vector<double>& h) {
    std::vector<DTYPE> t(h.begin(), h.end());
    DTYPE* d = nullptr;
    checkCudaErrors(cudaMalloc((void**)&d, sizeof(DTYPE) * (t.size() + 1)));
    checkCudaErrors(cudaMemcpy(d, t.data(), sizeof(DTYPE) * t.size(), cudaMemcpyHostToDevice));
    return d;
}

static DTYPE* dev_zeros(size_t n) {
    DTYPE* d = nullptr;
    checkCudaErrors(cudaMalloc((void**)&d, sizeof(DTYPE) * (n + 1)));
    checkCudaErrors(cudaMemset(d, 0, sizeof(DTYPE) * (n + 1)));
    return d;
}

static std::vector<double> from_dev(const DTYPE* d, size_t n) {
    std::vector<DTYPE> t(n);
    checkCudaErrors(cudaMemcpy(t.data(), d, sizeof(DTYPE) * n, cudaMemcpyDeviceToHost));
    return std::vector<double>(t.begin(), t.end());
}

static WaveletType wt(int id) { return static_cast<WaveletType>(id); }

int main(int argc, char** argv) {
    if (argc < 4) { fprintf(stderr, "usage: ref_driver op in_dir out_dir params...\n"); return 2; }
    std::string op = argv[1];
    g_in = argv[2];
    g_out = argv[3];
    auto I = [&](int k) { return atoi(argv[4 + k]); };
    auto D = [&](int k) { return atof(argv[4 + k]); };
    checkCudaErrors(cudaSetDevice(0));

    if (op == "dwt1d") {  // DX DY DZ levels axis bc wavelet fwd
        int3 dim = make_int3(I(0), I(1), I(2));
        size_t n = (size_t)dim.x * dim.y * dim.z;
        DTYPE* a = to_dev(read_bin("a", n));
        CuWHHDForward::GetInstance()->Solve1D(a, a, dim, I(3), argv[8][0], argv[9][0], wt(I(6)), I(7) != 0);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("c", from_dev(a, n));
    } else if (op == "ip") {  // dim wavelet bc
        int dim = I(0);
        DTYPE* ip = CuGetInnerProduct::GetInstance()->GenerateIp(wt(I(1)), argv[6][0], dim);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("ip", from_dev(ip, (size_t)dim * 8));
    } else if (op == "project3d" || op == "recover3d") {  // nx ny nz dx [bc]
        int3 dim = make_int3(I(0), I(1), I(2));
        DTYPE h = (DTYPE)D(3);
        const char wall = argc > 8 ? argv[8][0] : 'n';  // the walls' boundary type
        DTYPE3 dx = make_DTYPE3(h, h, h);
        size_t sxv = (size_t)(dim.x + 1) * dim.y * dim.z, syv = (size_t)dim.x * (dim.y + 1) * dim.z;
        size_t szv = (size_t)dim.x * dim.y * (dim.z + 1);
        size_t sqx = (size_t)dim.x * (dim.y + 1) * (dim.z + 1), sqy = (size_t)(dim.x + 1) * dim.y * (dim.z + 1);
        size_t sqz = (size_t)(dim.x + 1) * (dim.y + 1) * dim.z;
        DTYPE* xv = to_dev(read_bin("xv", sxv));
        DTYPE* yv = to_dev(read_bin("yv", syv));
        DTYPE* zv = to_dev(read_bin("zv", szv));
        DTYPE* qx = dev_zeros(sqx);
        DTYPE* qy = dev_zeros(sqy);
        DTYPE* qz = dev_zeros(sqz);
        int3 levels = make_int3((int)log2(dim.x), (int)log2(dim.y), (int)log2(dim.z));
        if (op == "project3d") {
            int3 dim_ext = make_int3(dim.x + 1, dim.y + 1, dim.z + 1);
            CuDivLocalProject3D cudlp(dim_ext, levels, dx, WaveletType::WT_CDF4_6, proj_bc(wall));
            cudlp.ProjectLocal_q_ccc(qx, qy, qz, xv, yv, zv, levels);
            checkCudaErrors(cudaGetLastError());
        } else {
            CuWaveletPotentialRecover3D rec(dim, dx, wall, WaveletType::WT_CDF3_7, WaveletType::WT_CDF4_6);
            rec.Solve(qx, qy, qz, xv, yv, zv);
        }
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("qx", from_dev(qx, sqx));
        write_bin("qy", from_dev(qy, sqy));
        write_bin("qz", from_dev(qz, sqz));
    } else if (op == "cut3d") {  // nx ny nz dx level: CuWaveletPotentialRecover3D::CutCoefficients
        int3 dim = make_int3(I(0), I(1), I(2));
        DTYPE h = (DTYPE)D(3);
        DTYPE3 dx = make_DTYPE3(h, h, h);
        int level = I(4);
        size_t sqx = (size_t)dim.x * (dim.y + 1) * (dim.z + 1), sqy = (size_t)(dim.x + 1) * dim.y * (dim.z + 1);
        size_t sqz = (size_t)(dim.x + 1) * (dim.y + 1) * dim.z;
        DTYPE* qx = to_dev(read_bin("qx", sqx));
        DTYPE* qy = to_dev(read_bin("qy", sqy));
        DTYPE* qz = to_dev(read_bin("qz", sqz));
        DTYPE* ox = dev_zeros(sqx);
        DTYPE* oy = dev_zeros(sqy);
        DTYPE* oz = dev_zeros(sqz);
        CuWaveletPotentialRecover3D rec(dim, dx, 'n', WaveletType::WT_CDF3_7, WaveletType::WT_CDF4_6);
        rec.CutCoefficients(ox, oy, oz, qx, qy, qz, level);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("qx", from_dev(ox, sqx));
        write_bin("qy", from_dev(oy, sqy));
        write_bin("qz", from_dev(oz, sqz));
    } else if (op == "frac3d_sub") {  // nx ny nz dx: static CuSolidLevelSet3D::GetFrac(ax, ay, az, ls, dim, dx)
        int3 dim = make_int3(I(0), I(1), I(2));
        DTYPE h = (DTYPE)D(3);
        DTYPE3 dx = make_DTYPE3(h, h, h);
        size_t n = (size_t)dim.x * dim.y * dim.z;
        size_t sx = (size_t)(dim.x + 1) * dim.y * dim.z, sy = (size_t)dim.x * (dim.y + 1) * dim.z;
        size_t sz = (size_t)dim.x * dim.y * (dim.z + 1);
        DTYPE* ls = to_dev(read_bin("ls", n));
        DTYPE* ax = dev_zeros(sx);
        DTYPE* ay = dev_zeros(sy);
        DTYPE* az = dev_zeros(sz);
        CuSolidLevelSet3D::GetFrac(ax, ay, az, ls, dim, dx);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("ax", from_dev(ax, sx));
        write_bin("ay", from_dev(ay, sy));
        write_bin("az", from_dev(az, sz));
    } else if (op == "fsweep") {  // nx ny nz dx iters reinit: CuFastSweeping::Solve / ReinitLevelSet
        int3 dim = make_int3(I(0), I(1), I(2));
        DTYPE h = (DTYPE)D(3);
        int iters = I(4), reinit = I(5);
        size_t n = (size_t)dim.x * dim.y * dim.z;
        DTYPE* ls = to_dev(read_bin("ls", n));
        if (reinit) CuFastSweeping::ReinitLevelSet(ls, dim, h, iters);
        else CuFastSweeping::Solve(ls, dim, h, iters);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("ls", from_dev(ls, n));
    } else if (op == "p2ls") {  // nx ny nz dx radius max_dis iters count: CuFastSweeping::ParticlesToLs
        int3 dim = make_int3(I(0), I(1), I(2));
        DTYPE h = (DTYPE)D(3), radius = (DTYPE)D(4), max_dis = (DTYPE)D(5);
        int iters = I(6), count = I(7);
        size_t n = (size_t)dim.x * dim.y * dim.z;
        DTYPE* x = to_dev(read_bin("xyz", (size_t)count * 3));
        DTYPE* ls = dev_zeros(n);
        CuFastSweeping::ParticlesToLs(ls, reinterpret_cast<DTYPE3*>(x), dim, count, h, radius, max_dis, iters);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("ls", from_dev(ls, n));
    } else if (op == "p2ls_narrow") {  // nx ny nz dx radius max_dis iters count: ParticlesToLsNarrow on ls
        int3 dim = make_int3(I(0), I(1), I(2));
        DTYPE h = (DTYPE)D(3), radius = (DTYPE)D(4), max_dis = (DTYPE)D(5);
        int iters = I(6), count = I(7);
        size_t n = (size_t)dim.x * dim.y * dim.z;
        DTYPE* x = to_dev(read_bin("xyz", (size_t)count * 3));
        DTYPE* ls = to_dev(read_bin("ls", n));
        CuFastSweeping::ParticlesToLsNarrow(ls, reinterpret_cast<DTYPE3*>(x), dim, count, h, radius, max_dis, iters);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("ls", from_dev(ls, n));
    } else if (op == "project2d" || op == "recover2d") {  // nx ny dx [bc [dy]]
        int2 dim = make_int2(I(0), I(1));
        DTYPE h = (DTYPE)D(2);
        const char wall = argc > 7 ? argv[7][0] : 'n';  // the walls' boundary type
        DTYPE2 dx = make_DTYPE2(h, argc > 8 ? (DTYPE)D(4) : h);
        size_t sxv = (size_t)(dim.x + 1) * dim.y, syv = (size_t)dim.x * (dim.y + 1), sqz = (size_t)(dim.x + 1) * (dim.y + 1);
        DTYPE* xv = to_dev(read_bin("xv", sxv));
        DTYPE* yv = to_dev(read_bin("yv", syv));
        DTYPE* qz = dev_zeros(sqz);
        int2 levels = make_int2((int)log2(dim.x), (int)log2(dim.y));
        if (op == "project2d") {
            int2 dim_ext = make_int2(dim.x + 1, dim.y + 1);
            CuDivLocalProject cudlp(dim_ext, levels, dx, WaveletType::WT_CDF4_6, proj_bc(wall));
            cudlp.ProjectSingle(qz, xv, yv);
            checkCudaErrors(cudaGetLastError());  // ProjectSingle does not check its own launch
        } else {
            CuWaveletPotentialRecover2D rec(dim, dx, wall, WaveletType::WT_CDF3_7, WaveletType::WT_CDF4_6);
            rec.Solve(qz, xv, yv);
        }
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("qz", from_dev(qz, sqz));
    } else if (op == "mg3d") {  // nx ny nz dx ncycles nu1 nu2 omega
        int3 dim = make_int3(I(0), I(1), I(2));
        DTYPE h = (DTYPE)D(3);
        DTYPE3 dx = make_DTYPE3(h, h, h);
        int ncycles = I(4), nu1 = I(5), nu2 = I(6);
        DTYPE w = (DTYPE)D(7);
        size_t n = (size_t)dim.x * dim.y * dim.z;
        DTYPE* f = to_dev(read_bin("f", n));
        DTYPE* ax = to_dev(read_bin("ax", (size_t)(dim.x + 1) * dim.y * dim.z));
        DTYPE* ay = to_dev(read_bin("ay", (size_t)dim.x * (dim.y + 1) * dim.z));
        DTYPE* az = to_dev(read_bin("az", (size_t)dim.x * dim.y * (dim.z + 1)));
        DTYPE* p = dev_zeros(n);
        CuMultigridFrac3D mg(ax, ay, az, dim, dx, 'n');
        std::vector<double> hist;
        for (int c = 0; c < ncycles; ++c) {
            mg.Solve(p, c == 0 ? nullptr : p, f, 1, nu1, nu2, w);
            hist.push_back((double)mg.GetResdualError(p, f));
        }
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("p", from_dev(p, n));
        write_bin("hist", hist);
    } else if (op == "mg3d_index") {  // nx ny nz dx ncycles nu1 nu2 omega [time_reps]
        // CuMultigridFrac3D::Solve_index one cycle per call (the residual workspace carries over
        // between calls, as between the cycles of one call); with time_reps > 0 also the best of
        // time_reps timed calls of ncycles cycles each, index-sparse and dense, on fresh iterates.
        int3 dim = make_int3(I(0), I(1), I(2));
        DTYPE h = (DTYPE)D(3);
        DTYPE3 dx = make_DTYPE3(h, h, h);
        int ncycles = I(4), nu1 = I(5), nu2 = I(6);
        DTYPE w = (DTYPE)D(7);
        int reps = argc > 12 ? I(8) : 0;
        size_t n = (size_t)dim.x * dim.y * dim.z;
        DTYPE* f = to_dev(read_bin("f", n));
        DTYPE* ax = to_dev(read_bin("ax", (size_t)(dim.x + 1) * dim.y * dim.z));
        DTYPE* ay = to_dev(read_bin("ay", (size_t)dim.x * (dim.y + 1) * dim.z));
        DTYPE* az = to_dev(read_bin("az", (size_t)dim.x * dim.y * (dim.z + 1)));
        DTYPE* p = dev_zeros(n);
        CuMultigridFrac3D mg(ax, ay, az, dim, dx, 'n');
        std::vector<double> hist;
        for (int c = 0; c < ncycles; ++c) {
            mg.Solve_index(p, c == 0 ? nullptr : p, f, 1, nu1, nu2, w);
            hist.push_back((double)mg.GetResdualError(p, f));
        }
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("p", from_dev(p, n));
        write_bin("hist", hist);
        if (reps > 0) {
            cudaEvent_t e0, e1;
            checkCudaErrors(cudaEventCreate(&e0));
            checkCudaErrors(cudaEventCreate(&e1));
            std::vector<double> best = {1e30, 1e30};
            for (int k = 0; k < 2; ++k)
                for (int r = 0; r < reps + 1; ++r) {
                    checkCudaErrors(cudaDeviceSynchronize());
                    checkCudaErrors(cudaEventRecord(e0));
                    if (k == 0) mg.Solve_index(p, nullptr, f, ncycles, nu1, nu2, w);
                    else mg.Solve(p, nullptr, f, ncycles, nu1, nu2, w);
                    checkCudaErrors(cudaEventRecord(e1));
                    checkCudaErrors(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    checkCudaErrors(cudaEventElapsedTime(&ms, e0, e1));
                    if (r > 0 && ms < best[k]) best[k] = ms;  // the first call of each is a warm-up
                }
            write_bin("timing", best);
        }
    } else if (op == "mg2d") {  // nx ny dx ncycles nu1 nu2 omega
        int2 dim = make_int2(I(0), I(1));
        DTYPE h = (DTYPE)D(2);
        DTYPE2 dx = make_DTYPE2(h, h);
        int ncycles = I(3), nu1 = I(4), nu2 = I(5);
        DTYPE w = (DTYPE)D(6);
        size_t n = (size_t)dim.x * dim.y;
        DTYPE* f = to_dev(read_bin("f", n));
        DTYPE* ax = to_dev(read_bin("ax", (size_t)(dim.x + 1) * dim.y));
        DTYPE* ay = to_dev(read_bin("ay", (size_t)dim.x * (dim.y + 1)));
        DTYPE* p = dev_zeros(n);
        std::vector<DTYPE> hdx(dim.x, h), hdy(dim.y, h);
        DTYPE *ddx = nullptr, *ddy = nullptr;
        checkCudaErrors(cudaMalloc((void**)&ddx, sizeof(DTYPE) * dim.x));
        checkCudaErrors(cudaMalloc((void**)&ddy, sizeof(DTYPE) * dim.y));
        checkCudaErrors(cudaMemcpy(ddx, hdx.data(), sizeof(DTYPE) * dim.x, cudaMemcpyHostToDevice));
        checkCudaErrors(cudaMemcpy(ddy, hdy.data(), sizeof(DTYPE) * dim.y, cudaMemcpyHostToDevice));
        CuMultigridFrac2D mg(ax, ay, dim, dx, 'n');
        std::vector<double> hist;
        for (int c = 0; c < ncycles; ++c) {
            mg.Solve(p, c == 0 ? nullptr : p, f, 1, nu1, nu2, w);
            hist.push_back((double)CuWeightedJacobi::GetFracRhs(p, f, ax, ay, dim, ddx, ddy, dx, 'n'));
        }
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("p", from_dev(p, n));
        write_bin("hist", hist);
    } else if (op == "div3d" || op == "grad3d") {  // nx ny nz dx
        int3 dim = make_int3(I(0), I(1), I(2));
        DTYPE h = (DTYPE)D(3);
        DTYPE3 dx = make_DTYPE3(h, h, h);
        size_t sxv = (size_t)(dim.x + 1) * dim.y * dim.z, syv = (size_t)dim.x * (dim.y + 1) * dim.z;
        size_t szv = (size_t)dim.x * dim.y * (dim.z + 1), n = (size_t)dim.x * dim.y * dim.z;
        DTYPE* xv = to_dev(read_bin("xv", sxv));
        DTYPE* yv = to_dev(read_bin("yv", syv));
        DTYPE* zv = to_dev(read_bin("zv", szv));
        DTYPE* ax = to_dev(read_bin("ax", sxv));
        DTYPE* ay = to_dev(read_bin("ay", syv));
        DTYPE* az = to_dev(read_bin("az", szv));
        if (op == "div3d") {
            DTYPE* b = dev_zeros(n);
            CuConvergence::GetInstance()->GetB_3d_frac_vel(b, xv, yv, zv, ax, ay, az, dim, dx, 'n');
            checkCudaErrors(cudaDeviceSynchronize());
            write_bin("b", from_dev(b, n));
        } else {
            DTYPE* p = to_dev(read_bin("p", n));
            std::vector<DTYPE> hx(dim.x, h), hy(dim.y, h), hz(dim.z, h);
            DTYPE *ddx = to_dev(std::vector<double>(dim.x, D(3))), *ddy = to_dev(std::vector<double>(dim.y, D(3)));
            DTYPE* ddz = to_dev(std::vector<double>(dim.z, D(3)));
            DTYPE* gx = dev_zeros(sxv);
            DTYPE* gy = dev_zeros(syv);
            DTYPE* gz = dev_zeros(szv);
            // TestLocalProjection.cpp:672-680: u <- a * (u - grad p)
            CuGradient::GetInstance()->Gradient3D_Frac_P(gx, gy, gz, p, ax, ay, az, dim, ddx, ddy, ddz, dx, 'n');
            CudaMatAdd(xv, gx, (int)sxv, -1.f);
            CudaMatAdd(yv, gy, (int)syv, -1.f);
            CudaMatAdd(zv, gz, (int)szv, -1.f);
            CudaMatMul(xv, xv, ax, (int)sxv);
            CudaMatMul(yv, yv, ay, (int)syv);
            CudaMatMul(zv, zv, az, (int)szv);
            checkCudaErrors(cudaDeviceSynchronize());
            write_bin("xv", from_dev(xv, sxv));
            write_bin("yv", from_dev(yv, syv));
            write_bin("zv", from_dev(zv, szv));
        }
    } else if (op == "frac3d") {  // n dx cx cy cz r
        int n = I(0);
        int3 dim = make_int3(n, n, n);
        DTYPE h = (DTYPE)D(1);
        DTYPE3 dx = make_DTYPE3(h, h, h);
        size_t sf = (size_t)(n + 1) * n * n;
        DTYPE* ax = dev_zeros(sf);
        DTYPE* ay = dev_zeros(sf);
        DTYPE* az = dev_zeros(sf);
        CuSolidLevelSet3D sls(dim, dx);
        sls.InitLsSphere(make_DTYPE3((DTYPE)D(2), (DTYPE)D(3), (DTYPE)D(4)), (DTYPE)D(5));
        sls.GetFrac(ax, ay, az);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("ax", from_dev(ax, sf));
        write_bin("ay", from_dev(ay, sf));
        write_bin("az", from_dev(az, sf));
    } else if (op == "dst3d") {  // nx ny nz dx dy dz: CuDst3D(dim, dx).Solve(p, f)
        // equal extents only: the constructor sizes its buffer as the largest of the x and z FFT
        // layouts and a member it never sets (cuDst3D.cu:209-211); with equal extents every layout
        // has the same size, so the buffer always holds the y pass too
        int3 dim = make_int3(I(0), I(1), I(2));
        if (dim.x != dim.y || dim.y != dim.z) { fprintf(stderr, "dst3d: equal extents only\n"); return 2; }
        DTYPE3 dx = make_DTYPE3((DTYPE)D(3), (DTYPE)D(4), (DTYPE)D(5));
        size_t nc = (size_t)dim.x * dim.y * dim.z;
        DTYPE* f = to_dev(read_bin("f", nc));
        DTYPE* p = dev_zeros(nc);
        CuDst3D dst(dim, dx);
        dst.Solve(p, f);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("p", from_dev(p, nc));
    } else if (op == "psweep3d") {  // n dx [bc [solve_only]]: CuParallelSweep3D(dim, dx, bc) Solve, then Project
        // (TestLocalProjection.cpp:719-721); equal extents only (its CuDst3D on the (n-1)^3 nodes).  With
        // solve_only = 1 Project is not called (its bc 'd' branch, ProjectD, raised an illegal address
        // at 16^3 and is not run)
        const char wall = argc > 6 ? argv[6][0] : 'n';
        const bool solve_only = argc > 7 && atoi(argv[7]) != 0;
        int n = I(0);
        int3 dim = make_int3(n, n, n);
        DTYPE h = (DTYPE)D(1);
        DTYPE3 dx = make_DTYPE3(h, h, h);
        size_t sf = (size_t)(n + 1) * n * n, sq = (size_t)n * (n + 1) * (n + 1);
        DTYPE* xv = to_dev(read_bin("xv", sf));
        DTYPE* yv = to_dev(read_bin("yv", sf));
        DTYPE* zv = to_dev(read_bin("zv", sf));
        DTYPE *qx = dev_zeros(sq), *qy = dev_zeros(sq), *qz = dev_zeros(sq);
        CuParallelSweep3D cups(dim, dx, wall);
        cups.Solve(qx, qy, qz, xv, yv, zv);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("qx_solve", from_dev(qx, sq));
        write_bin("qy_solve", from_dev(qy, sq));
        write_bin("qz_solve", from_dev(qz, sq));
        if (solve_only) return 0;
        cups.Project(qx, qy, qz);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("qx", from_dev(qx, sq));
        write_bin("qy", from_dev(qy, sq));
        write_bin("qz", from_dev(qz, sq));
    } else if (op == "psweep3d_mid") {  // n dx mx my mz: CuParallelSweep3D(dim, dx, 'n').SolveFromMid(..., mid)
        int n = I(0);
        int3 dim = make_int3(n, n, n);
        DTYPE h = (DTYPE)D(1);
        DTYPE3 dx = make_DTYPE3(h, h, h);
        int3 mid = make_int3(I(2), I(3), I(4));
        size_t sf = (size_t)(n + 1) * n * n, sq = (size_t)n * (n + 1) * (n + 1);
        DTYPE* xv = to_dev(read_bin("xv", sf));
        DTYPE* yv = to_dev(read_bin("yv", sf));
        DTYPE* zv = to_dev(read_bin("zv", sf));
        DTYPE *qx = dev_zeros(sq), *qy = dev_zeros(sq), *qz = dev_zeros(sq);
        CuParallelSweep3D cups(dim, dx, 'n');
        cups.SolveFromMid(qx, qy, qz, xv, yv, zv, mid);
        checkCudaErrors(cudaGetLastError());
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("qx", from_dev(qx, sq));
        write_bin("qy", from_dev(qy, sq));
        write_bin("qz", from_dev(qz, sq));
    } else if (op == "psweep2d") {  // n dx [bc]: CuParallelSweep3D(int2 dim, DTYPE2 dx, bc).Solve(qz, xv, yv)
        const char wall = argc > 6 ? argv[6][0] : 'n';
        int n = I(0);
        DTYPE h = (DTYPE)D(1);
        size_t sf = (size_t)(n + 1) * n, sq = (size_t)(n + 1) * (n + 1);
        DTYPE* xv = to_dev(read_bin("xv", sf));
        DTYPE* yv = to_dev(read_bin("yv", sf));
        DTYPE* qz = dev_zeros(sq);
        CuParallelSweep3D cups(make_int2(n, n), make_DTYPE2(h, h), wall);
        cups.Solve(qz, xv, yv);
        checkCudaErrors(cudaDeviceSynchronize());
        write_bin("qz", from_dev(qz, sq));
    } else if (op == "bench3d") {  // n ncycles nu1 nu2 omega reps : one projection per rep, CUDA events
        int n = I(0), ncycles = I(1), nu1 = I(2), nu2 = I(3), reps = I(5);
        DTYPE w = (DTYPE)D(4);
        int3 dim = make_int3(n, n, n);
        DTYPE h = (DTYPE)(1.0 / n);
        DTYPE3 dx = make_DTYPE3(h, h, h);
        size_t sf = (size_t)(n + 1) * n * n, nc = (size_t)n * n * n;
        DTYPE* xv = to_dev(read_bin("xv", sf));
        DTYPE* yv = to_dev(read_bin("yv", sf));
        DTYPE* zv = to_dev(read_bin("zv", sf));
        DTYPE* ax = to_dev(read_bin("ax", sf));
        DTYPE* ay = to_dev(read_bin("ay", sf));
        DTYPE* az = to_dev(read_bin("az", sf));
        DTYPE *ux = dev_zeros(sf), *uy = dev_zeros(sf), *uz = dev_zeros(sf);
        DTYPE *gx = dev_zeros(sf), *gy = dev_zeros(sf), *gz = dev_zeros(sf);
        DTYPE *qx = dev_zeros(sf + n * n + n), *qy = dev_zeros(sf + n * n + n), *qz = dev_zeros(sf + n * n + n);
        DTYPE *f = dev_zeros(nc), *p = dev_zeros(nc), *b = dev_zeros(nc);
        DTYPE *ddx = to_dev(std::vector<double>(n, 1.0 / n));
        CuMultigridFrac3D mg(ax, ay, az, dim, dx, 'n');
        CuWaveletPotentialRecover3D rec(dim, dx, 'n', WaveletType::WT_CDF3_7, WaveletType::WT_CDF4_6);
        cudaEvent_t e0, e1, es, eg;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventCreate(&es);
        cudaEventCreate(&eg);
        double best = 1e30, total = 0.0, maxdiv = 0.0, relres = 0.0, t_solve = 0.0, t_grad = 0.0, t_rec = 0.0;
        for (int r = 0; r < reps + 1; ++r) {
            checkCudaErrors(cudaMemcpy(ux, xv, sizeof(DTYPE) * sf, cudaMemcpyDeviceToDevice));
            checkCudaErrors(cudaMemcpy(uy, yv, sizeof(DTYPE) * sf, cudaMemcpyDeviceToDevice));
            checkCudaErrors(cudaMemcpy(uz, zv, sizeof(DTYPE) * sf, cudaMemcpyDeviceToDevice));
            checkCudaErrors(cudaDeviceSynchronize());
            cudaEventRecord(e0);
            CuConvergence::GetInstance()->GetB_3d_frac_vel(f, ux, uy, uz, ax, ay, az, dim, dx, 'n');
            mg.Solve(p, nullptr, f, ncycles, nu1, nu2, w);
            cudaEventRecord(es);
            CuGradient::GetInstance()->Gradient3D_Frac_P(gx, gy, gz, p, ax, ay, az, dim, ddx, ddx, ddx, dx, 'n');
            CudaMatAdd(ux, gx, (int)sf, -1.f);
            CudaMatAdd(uy, gy, (int)sf, -1.f);
            CudaMatAdd(uz, gz, (int)sf, -1.f);
            CuConvergence::GetInstance()->GetB_3d_frac_vel(b, ux, uy, uz, ax, ay, az, dim, dx, 'n');
            maxdiv = (double)CudaFindMaxValue(b, (int)nc);
            CudaMatMul(ux, ux, ax, (int)sf);
            CudaMatMul(uy, uy, ay, (int)sf);
            CudaMatMul(uz, uz, az, (int)sf);
            cudaEventRecord(eg);
            rec.Solve(qx, qy, qz, ux, uy, uz);
            cudaEventRecord(e1);
            checkCudaErrors(cudaEventSynchronize(e1));
            float ms = 0.f, m0 = 0.f, m1 = 0.f, m2 = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            cudaEventElapsedTime(&m0, e0, es);
            cudaEventElapsedTime(&m1, es, eg);
            cudaEventElapsedTime(&m2, eg, e1);
            if (r > 0) {
                total += ms;
                if (ms < best) best = ms;
                t_solve += m0;
                t_grad += m1;
                t_rec += m2;
            }
        }
        relres = (double)mg.GetResdualError(p, f);
        printf("{\"n\": %d, \"ncycles\": %d, \"nu1\": %d, \"nu2\": %d, \"omega\": %g, \"reps\": %d, \"ms_best\": %.4f, "
               "\"ms_mean\": %.4f, \"ms_divergence_and_solve\": %.4f, \"ms_gradient_update_maxdiv\": %.4f, "
               "\"ms_recovery\": %.4f, \"rel_residual\": %.3e, \"max_abs_div\": %.3e, \"dtype_bytes\": %d}\n",
               n, ncycles, nu1, nu2, (double)w, reps, best, total / reps, t_solve / reps, t_grad / reps, t_rec / reps,
               relres, maxdiv, (int)sizeof(DTYPE));
    } else {
        fprintf(stderr, "unknown op %s\n", op.c_str());
        return 2;
    }
    return 0;
}
