// wp_mg_fused.cuh -- one level of the FP32 V(2,2) cycle in two kernels with temporal blocking
// (included by wp_mg.cu inside its anonymous namespace, after Lvl / Q4 and the quad helpers).
//
//   cycle_down_kernel: two weighted-Jacobi pre-sweeps (the first from zero, or from the level's
//     iterate), the residual f - A v and its restriction to the coarse right-hand side
//     (cuWjFrac3D_n x 2 + cuWjGetFracRes_3d_n + cuRestrict3D_p1_d{x,y,z}: cuWeightedJacobi3D.cu:620-695,
//     1107-1181, cuRestrict3D.cu:801-970);
//   cycle_up_kernel: the cell-centred trilinear prolongation of the coarse correction added to the
//     iterate, then two post-sweeps, the result stored or added to the FP64 iterate of the
//     mixed-precision refinement.
//
// Each costs one pass over the level instead of three: the down kernel reads f (and the iterate)
// and writes the swept iterate and the coarse right-hand side; the up kernel reads the iterate, f
// and the coarse correction and writes the result.  The per-cell arithmetic is that of the one-sweep
// kernels (QCol::step_with / jacobi0_q_body / resid_restrict_q_body / prolong_tri_q_body): same
// terms in the same order, except that on uniform planes the update multiplies by a precomputed
// w / diagonal instead of dividing by the diagonal.
//
// Scheme.  A CTA owns an output tile of TY (y) x TX (x) cells and a z-chunk.  Its 384 threads each
// own one y-quad column of the first stage's region (the tile with a 4-cell y halo and a 2-cell x
// halo) and march up z with three stages in flight: stage 1 at plane t (first sweep / prolongation,
// over the whole region), stage 2 at plane t - 1 (second sweep, one cell of x halo) and stage 3 at
// plane t - 2 (residual + restriction / second post-sweep, the tile).  A stage's x/y neighbours come
// from the previous stage's plane in shared memory, its z neighbours and its own centre from the
// thread's registers (the column is the same at every stage); two block barriers per plane.  The
// input planes (iterate with a 3-cell x halo, f) stream in through TMA tile loads into a 6-plane
// ring (out-of-range elements read as zero), issued four planes ahead by one thread.  Stencil
// coefficients: the per-axis spacing factors, times the face fractions on tile-planes that are
// not uniform (fractions read through L1 there; a per (plane, tile) flag built with the level).
// Cells outside the level get zero coefficients, so their values are 0 and never reach a result.

namespace fz {
constexpr int TY = 32, TX = 32;          // output tile (y by x cells)
constexpr int RY = TY + 8, RX = TX + 4;  // first-stage region: y halo 4 (whole quads), x halo 2
constexpr int NQ = RY / 4;               // quads per region row
constexpr int NIN = (TX * TY) / 4;       // quad columns of the output tile (threads 0 .. NIN-1)
constexpr int NCOL = NQ * RX;            // quad columns of the region, one per thread
constexpr int THREADS = 384;
constexpr int PL = RY * RX;              // floats of one stage plane
constexpr int VPL = 1536;                // floats of one iterate plane (RX + 2 rows, padded to 128 B)
constexpr int SLOT = VPL + PL;           // one plane of the input stream: iterate, then f
constexpr int SLOTS = 8;                 // planes in the ring (two are consumed per iteration)
constexpr int SB = 4;                    // stage planes kept per stage (two written, two read per iteration)
constexpr int ZT = 256;                  // plane-table entries: a chunk holds at most ZT - 6 planes
constexpr size_t smem_floats = (size_t)SLOTS * SLOT + 2 * SB * PL + 2 * RX + 2 * RY + 4 * ZT;
constexpr size_t smem_bytes = smem_floats * 4 + SLOTS * 8;
static_assert(NCOL <= THREADS && NIN % 32 == 0, "one thread per quad column, the tile's in whole warps");
static_assert((VPL * 4) % 128 == 0 && (PL * 4) % 128 == 0, "TMA destinations stay 128-byte aligned");
static_assert((RX + 2) * RY <= VPL, "the iterate plane holds a 3-cell x halo");
static_assert((smem_floats * 4) % 8 == 0, "mbarriers are 8-byte aligned");
// plane modes
constexpr int IN = 1;    // the plane lies in the level
constexpr int UNI = 2;   // every interior face fraction of the tile's region on it is 1
constexpr int STD = 4;   // its z factors are those of the reference interior plane, and every diagonal
                         // of such a plane is positive (the straight-line path)
constexpr int FAST = IN | UNI | STD;
}  // namespace fz

// One plane of a CTA's chunk: z factors, restriction weight and mode (plane table in shared memory)
struct FzPlane {
    float gzl, gzh, wz;
    int mode;
};
__device__ __forceinline__ bool fz_fast(const FzPlane& P) { return (P.mode & fz::FAST) == fz::FAST; }

// One thread's quad column of the region, its spacing factors (0 outside the level) and, for the
// straight-line path, each cell's diagonal and w / diagonal with the reference z factors.
struct FzCol {
    int xr, q, o, ov;  // region row and quad; offset in a stage plane and in an iterate plane
    int x, yq;         // level coordinates of the quad's first cell
    bool r1, r2;       // the column takes part in stage 1 / 2 (stage 3: the output tile, tid < NIN)
    bool cin;          // the quad lies inside the level
    float gxl, gxh, gyl[4], gyh[4];
    float dstd[4], wdstd[4];
};

// the per-axis face factors of the region's rows and columns (0 outside the level) and the plane
// table of planes pb .. pb + np - 1; fast_ok: the level's diagonals are positive on uniform planes
// with the reference z factors (checked on the host when the level is built)
__device__ __forceinline__ void fz_tables(const Lvl<float>& L, int x0, int y0, float* gxs, float* gys, FzPlane* pz,
                                          int pb, int np, const unsigned char* __restrict__ tuni, int ntiles, int tile,
                                          int fast_ok, int tid) {
    for (int j = tid; j < fz::RX; j += fz::THREADS) {
        const int x = x0 - 2 + j;
        const bool in = x >= 0 && x < L.nx;
        gxs[j] = in ? L.glo[0][x] : 0.f;
        gxs[fz::RX + j] = in ? L.ghi[0][x] : 0.f;
    }
    for (int j = tid; j < fz::RY; j += fz::THREADS) {
        const int y = y0 - 4 + j;
        const bool in = y >= 0 && y < L.ny;
        gys[j] = in ? L.glo[1][y] : 0.f;
        gys[fz::RY + j] = in ? L.ghi[1][y] : 0.f;
    }
    const int zr = L.nz / 2;
    const float rl = L.glo[2][zr], rh = L.ghi[2][zr];
    for (int j = tid; j < np; j += fz::THREADS) {
        const int p = pb + j;
        FzPlane e{0.f, 0.f, 0.f, 0};
        if (p >= 0 && p < L.nz) {
            e.gzl = L.glo[2][p];
            e.gzh = L.ghi[2][p];
            const int zb = p & ~1;
            e.wz = zb + 1 < L.nz ? (float)(L.d[2][p] / (L.d[2][zb] + L.d[2][zb + 1])) : 0.f;
            e.mode = fz::IN | (tuni[(long)p * ntiles + tile] ? fz::UNI : 0) |
                     (fast_ok && e.gzl == rl && e.gzh == rh ? fz::STD : 0);
        }
        pz[j] = e;
    }
}

// Thread -> quad column: threads 0 .. NIN-1 own the output tile (8 quads per region row, 4 rows
// per warp, so the x-pair of a coarse cell is lanes l and l + 8 of one warp), the next ones the
// halo: the two region rows on each x side, then the first and last quad of every tile row.
__device__ __forceinline__ FzCol fz_column(const Lvl<float>& L, int x0, int y0, const float* gxs, const float* gys,
                                           float w, int tid) {
    using namespace fz;
    FzCol c;
    c.r1 = tid < NCOL;
    if (tid < NIN) {
        c.xr = 2 + tid / (TY / 4);
        c.q = 1 + tid % (TY / 4);
    } else if (tid < NIN + 4 * NQ) {
        const int j = tid - NIN;
        c.xr = j < 2 * NQ ? j / NQ : RX - 4 + j / NQ;
        c.q = j % NQ;
    } else if (tid < NCOL) {
        const int j = tid - NIN - 4 * NQ;
        c.xr = 2 + j / 2;
        c.q = (j & 1) ? NQ - 1 : 0;
    } else {
        c.xr = 0;
        c.q = 0;
    }
    c.r2 = c.r1 && c.xr >= 1 && c.xr < RX - 1;
    c.o = c.xr * RY + 4 * c.q;
    c.ov = c.o + RY;
    c.x = x0 - 2 + c.xr;
    c.yq = y0 - 4 + 4 * c.q;
    c.cin = c.r1 && c.x >= 0 && c.x < L.nx && c.yq >= 0 && c.yq < L.ny;
    c.gxl = gxs[c.xr];
    c.gxh = gxs[RX + c.xr];
    const int zr = L.nz / 2;
    const float rl = L.glo[2][zr], rh = L.ghi[2][zr];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        c.gyl[k] = gys[4 * c.q + k];
        c.gyh[k] = gys[RY + 4 * c.q + k];
        // the diagonal summed in the general path's order (y, x, z faces)
        const float d = ((((c.gyl[k] + c.gyh[k]) + c.gxl) + c.gxh) + rl) + rh;
        c.dstd[k] = d;
        c.wdstd[k] = d > (float)kEps ? w / d : 0.f;
    }
    return c;
}

// ---- general path: face fractions where the plane is not uniform, divisions, zero diagonals

// The six face coefficients (y lower/upper, x lower/upper, z lower/upper) of the quad's cells at
// plane z: spacing factor times face fraction (the fraction is 1 on a uniform tile-plane).
__device__ __forceinline__ void fz_coefs(const Lvl<float>& L, const FzCol& c, int z, const FzPlane& P,
                                         Q4<float> (&cf)[6]) {
    if (P.mode & fz::UNI) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            cf[0].a[k] = c.gyl[k];
            cf[1].a[k] = c.gyh[k];
            cf[2].a[k] = c.gxl;
            cf[3].a[k] = c.gxh;
            cf[4].a[k] = P.gzl;
            cf[5].a[k] = P.gzh;
        }
    } else {
        const int ny = L.ny;
        const long sxy = (long)L.nx * ny;
        const long i = c.yq + (long)c.x * ny + z * sxy;
        const long iax = c.yq + (long)c.x * ny + z * (long)(L.nx + 1) * ny;
        const Q4<float> fyl = ld4(L.fyc + i);
        const float fyu = c.yq + 4 < ny ? L.fyc[i + 4] : 0.f;
        const Q4<float> fxl = ld4(L.ax + iax), fxu = ld4(L.ax + iax + ny);
        const Q4<float> azl = ld4(L.az + i), azu = ld4(L.az + i + sxy);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            cf[0].a[k] = fyl.a[k] * c.gyl[k];
            cf[1].a[k] = (k < 3 ? fyl.a[k + 1] : fyu) * c.gyh[k];
            cf[2].a[k] = fxl.a[k] * c.gxl;
            cf[3].a[k] = fxu.a[k] * c.gxh;
            cf[4].a[k] = azl.a[k] * P.gzl;
            cf[5].a[k] = azu.a[k] * P.gzh;
        }
    }
}

// diagonal and off-diagonal sum A v = dg v - od of the quad (QCol::step_with's terms and order)
__device__ __forceinline__ void fz_row(const Q4<float> (&cf)[6], const Q4<float>& c, float ym, float yp,
                                       const Q4<float>& xm, const Q4<float>& xp, const Q4<float>& zm,
                                       const Q4<float>& zp, Q4<float>& dg, Q4<float>& od) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float d = 0.f, o = 0.f, cv;
        cv = cf[0].a[k]; d += cv; o -= cv * (k > 0 ? c.a[k - 1] : ym);
        cv = cf[1].a[k]; d += cv; o -= cv * (k < 3 ? c.a[k + 1] : yp);
        cv = cf[2].a[k]; d += cv; o -= cv * xm.a[k];
        cv = cf[3].a[k]; d += cv; o -= cv * xp.a[k];
        cv = cf[4].a[k]; d += cv; o -= cv * zm.a[k];
        cv = cf[5].a[k]; d += cv; o -= cv * zp.a[k];
        dg.a[k] = d;
        od.a[k] = o;
    }
}

// ---- straight-line path: a uniform plane with the reference z factors, positive diagonals

__device__ __forceinline__ Q4<float> fz_off_fast(const FzCol& c, float gzl, float gzh, const Q4<float>& v, float ym,
                                                 float yp, const Q4<float>& xm, const Q4<float>& xp,
                                                 const Q4<float>& zm, const Q4<float>& zp) {
    Q4<float> od;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float o = 0.f;
        o -= c.gyl[k] * (k > 0 ? v.a[k - 1] : ym);
        o -= c.gyh[k] * (k < 3 ? v.a[k + 1] : yp);
        o -= c.gxl * xm.a[k];
        o -= c.gxh * xp.a[k];
        o -= gzl * zm.a[k];
        o -= gzh * zp.a[k];
        od.a[k] = o;
    }
    return od;
}

__device__ __forceinline__ Q4<float> fz_sweep_fast(const FzCol& c, const FzPlane& P, const Q4<float>& v, float ym,
                                                   float yp, const Q4<float>& xm, const Q4<float>& xp,
                                                   const Q4<float>& zm, const Q4<float>& zp, const Q4<float>& f,
                                                   float omw) {
    const Q4<float> od = fz_off_fast(c, P.gzl, P.gzh, v, ym, yp, xm, xp, zm, zp);
    Q4<float> out;
#pragma unroll
    for (int k = 0; k < 4; ++k) out.a[k] = omw * v.a[k] + c.wdstd[k] * (f.a[k] - od.a[k]);
    return out;
}

__device__ __forceinline__ Q4<float> fz_resid_fast(const FzCol& c, const FzPlane& P, const Q4<float>& v, float ym,
                                                   float yp, const Q4<float>& xm, const Q4<float>& xp,
                                                   const Q4<float>& zm, const Q4<float>& zp, const Q4<float>& f) {
    const Q4<float> od = fz_off_fast(c, P.gzl, P.gzh, v, ym, yp, xm, xp, zm, zp);
    Q4<float> r;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.a[k] = f.a[k] - (c.dstd[k] * v.a[k] + od.a[k]);
    return r;
}

// ---- either path, chosen per plane

// One weighted-Jacobi sweep of the quad (0 on a plane outside the level)
__device__ __forceinline__ Q4<float> fz_sweep(const Lvl<float>& L, const FzCol& c, int z, const FzPlane& P,
                                              const Q4<float>& v, float ym, float yp, const Q4<float>& xm,
                                              const Q4<float>& xp, const Q4<float>& zm, const Q4<float>& zp,
                                              const Q4<float>& f, float w) {
    if (fz_fast(P)) return fz_sweep_fast(c, P, v, ym, yp, xm, xp, zm, zp, f, 1.f - w);
    Q4<float> out = zero4<float>();
    if (!(P.mode & fz::IN)) return out;
    Q4<float> cf[6], dg, od;
    fz_coefs(L, c, z, P, cf);
    fz_row(cf, v, ym, yp, xm, xp, zm, zp, dg, od);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        out.a[k] = dg.a[k] > (float)kEps ? (1.f - w) * v.a[k] + w * (f.a[k] - od.a[k]) / dg.a[k] : 0.f;
    return out;
}

// the first sweep from v = 0 (jacobi0_q_body): w f / diagonal
__device__ __forceinline__ Q4<float> fz_sweep0(const Lvl<float>& L, const FzCol& c, int z, const FzPlane& P,
                                               const Q4<float>& f, float w) {
    Q4<float> out = zero4<float>();
    if (fz_fast(P)) {
#pragma unroll
        for (int k = 0; k < 4; ++k) out.a[k] = c.wdstd[k] * f.a[k];
        return out;
    }
    if (!(P.mode & fz::IN)) return out;
    Q4<float> cf[6];
    fz_coefs(L, c, z, P, cf);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float d = ((((cf[0].a[k] + cf[1].a[k]) + cf[2].a[k]) + cf[3].a[k]) + cf[4].a[k]) + cf[5].a[k];
        out.a[k] = d > (float)kEps ? (1.f - w) * 0.f + w * (f.a[k] - 0.f) / d : 0.f;
    }
    return out;
}

// residual f - A v of the quad (0 where the diagonal is not positive)
__device__ __forceinline__ Q4<float> fz_resid(const Lvl<float>& L, const FzCol& c, int z, const FzPlane& P,
                                              const Q4<float>& v, float ym, float yp, const Q4<float>& xm,
                                              const Q4<float>& xp, const Q4<float>& zm, const Q4<float>& zp,
                                              const Q4<float>& f) {
    if (fz_fast(P)) return fz_resid_fast(c, P, v, ym, yp, xm, xp, zm, zp, f);
    Q4<float> cf[6], dg, od, r;
    fz_coefs(L, c, z, P, cf);
    fz_row(cf, v, ym, yp, xm, xp, zm, zp, dg, od);
#pragma unroll
    for (int k = 0; k < 4; ++k) r.a[k] = dg.a[k] > (float)kEps ? f.a[k] - (dg.a[k] * v.a[k] + od.a[k]) : 0.f;
    return r;
}

// prolong_tri_q_body's increments for the quad (x, y0..y0+3) at the planes A (even) and A + 1,
// which share their parent coarse plane: the y interpolation of each coarse row, then x, then z,
// the same products and sums as prolong_tri_q_body
__device__ __forceinline__ void fz_prolong2(const float* __restrict__ vc, int x, int y0, int A, int ncx, int ncy,
                                            int ncz, Q4<float>& inc_a, Q4<float>& inc_b) {
    const int px = x >> 1, pz = A >> 1;
    int qx = (x & 1) ? px + 1 : px - 1;
    if (qx < 0 || qx >= ncx) qx = px;
    const int qza = pz - 1 < 0 ? pz : pz - 1, qzb = pz + 1 >= ncz ? pz : pz + 1;
    const long sc = (long)ncx * ncy;
    const float a = 0.75f, b = 0.25f;
    const int cy0 = y0 >> 1;
    // y-interpolated values of the coarse row (xx, zz) for the quad's four cells
    auto yrow = [&](int xx, int zz) -> Q4<float> {
        const float* r = vc + cy0 + (long)xx * ncy + zz * sc;
        const float ra = __ldg(r), rb = __ldg(r + 1);
        const float rm = cy0 > 0 ? __ldg(r - 1) : ra;
        const float rp = cy0 + 2 < ncy ? __ldg(r + 2) : rb;
        Q4<float> o;
        o.a[0] = a * ra + b * rm;
        o.a[1] = a * ra + b * rb;
        o.a[2] = a * rb + b * ra;
        o.a[3] = a * rb + b * rp;
        return o;
    };
    const Q4<float> y00 = yrow(px, pz), y10 = yrow(qx, pz);
    const Q4<float> y0a = yrow(px, qza), y1a = yrow(qx, qza);
    const Q4<float> y0b = yrow(px, qzb), y1b = yrow(qx, qzb);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float lo = a * y00.a[k] + b * y10.a[k];
        const float ha = a * y0a.a[k] + b * y1a.a[k];
        const float hb = a * y0b.a[k] + b * y1b.a[k];
        inc_a.a[k] = a * lo + b * ha;
        inc_b.a[k] = a * lo + b * hb;
    }
}

// Shared-memory layout and the TMA input stream of both kernels.
struct FzSmem {
    float* ring;   // SLOTS x [iterate plane | f plane]
    float* b1;     // stage-1 planes, SB buffers
    float* b2;     // stage-2 planes, SB buffers
    float* gxs;    // x factors of the region (lower | upper)
    float* gys;    // y factors of the region (lower | upper)
    FzPlane* pz;   // plane table of the chunk
    unsigned long long* bars;
};

__device__ __forceinline__ FzSmem fz_smem(float* base) {
    using namespace fz;
    FzSmem m;
    m.ring = base;
    m.b1 = m.ring + SLOTS * SLOT;
    m.b2 = m.b1 + SB * PL;
    m.gxs = m.b2 + SB * PL;
    m.gys = m.gxs + 2 * RX;
    m.pz = reinterpret_cast<FzPlane*>(m.gys + 2 * RY);
    m.bars = reinterpret_cast<unsigned long long*>(m.gys + 2 * RY + 4 * ZT);
    return m;
}

// Input planes pb, pb + 1, ... of the CTA: plane p lives in slot (p - pb) % SLOTS; with_v: the
// iterate's rows x0-3 .. x0+34 are loaded too (box RY x RX+2), f's rows x0-2 .. x0+33 always.
struct FzStream {
    const CUtensorMap* mv;
    const CUtensorMap* mf;
    float* ring;
    unsigned long long* bars;
    int pb, pe, x0, y0;
    bool with_v;
    __device__ __forceinline__ float* slot(int p) const { return ring + ((p - pb) & (fz::SLOTS - 1)) * fz::SLOT; }
    __device__ __forceinline__ void issue(int p) const {
        if (p > pe) return;
        const uint32_t bar = wptc::smem_u32(&bars[(p - pb) & (fz::SLOTS - 1)]);
        float* d = slot(p);
        wptc::mbar_expect_tx(bar, (with_v ? (uint32_t)((fz::RX + 2) * fz::RY * 4) : 0u) + (uint32_t)(fz::PL * 4));
        if (with_v) wptc::tma_load_3d(wptc::smem_u32(d), mv, bar, y0 - 4, x0 - 3, p);
        wptc::tma_load_3d(wptc::smem_u32(d + fz::VPL), mf, bar, y0 - 4, x0 - 2, p);
    }
    __device__ __forceinline__ bool wait(int p, int* err) const {
        const int k = p - pb;
        return wptc::mbar_wait(wptc::smem_u32(&bars[k & (fz::SLOTS - 1)]), (uint32_t)((k / fz::SLOTS) & 1), err);
    }
};
static_assert((fz::SLOTS & (fz::SLOTS - 1)) == 0, "the ring's slot index is a mask");

// x/y neighbours of the quad in a stage plane (y ends of the region read 0)
struct FzNb {
    float ym, yp;
    Q4<float> xm, xp;
};
__device__ __forceinline__ FzNb fz_nb(const float* pl, int o, int q) {
    FzNb n;
    n.ym = q > 0 ? pl[o - 1] : 0.f;
    n.yp = q < fz::NQ - 1 ? pl[o + 4] : 0.f;
    n.xm = ld4(pl + o - fz::RY);
    n.xp = ld4(pl + o + fz::RY);
    return n;
}
// the same for a quad of the output tile (never at the region's y ends)
__device__ __forceinline__ FzNb fz_nb_in(const float* pl, int o) {
    FzNb n;
    n.ym = pl[o - 1];
    n.yp = pl[o + 4];
    n.xm = ld4(pl + o - fz::RY);
    n.xp = ld4(pl + o + fz::RY);
    return n;
}
__device__ __forceinline__ float* fz_stage(float* b, int p) { return b + (p & (fz::SB - 1)) * fz::PL; }

// Pre-smoothing + residual restriction.  ZERO: the iterate is 0 (no iterate stream).  dst receives
// the iterate after two sweeps on the tile's cells; fc the coarse right-hand side.  Each iteration
// advances two planes: stage 1 at planes A, A+1, stage 2 at A-1, A, stage 3 (a whole coarse plane)
// at A-2, A-1, for A = z0-2, z0, ..., z1.
template <bool ZERO>
__global__ void __launch_bounds__(fz::THREADS, 1)
    cycle_down_kernel(const __grid_constant__ CUtensorMap mv, const __grid_constant__ CUtensorMap mf,
                      float* __restrict__ dst, float* __restrict__ fc, Lvl<float> L,
                      const unsigned char* __restrict__ tuni, float w, int zc, int fast_ok, int* __restrict__ err) {
    using namespace fz;
    extern __shared__ __align__(128) float fz_raw[];
    const FzSmem sm = fz_smem(fz_raw);
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const int nty = ny / TY, ntiles = nty * (nx / TX);
    const int tile = blockIdx.x, x0 = (tile / nty) * TX, y0 = (tile - (tile / nty) * nty) * TY;
    const int z0 = blockIdx.y * zc, z1 = min(z0 + zc, nz);
    const int tid = threadIdx.x;
    const bool tin = tid < NIN;  // the thread owns a quad of the output tile (whole warps)
    const int ncx = nx >> 1, ncy = ny >> 1;
    const long sxy = (long)nx * ny, csxy = (long)ncx * ncy;
    const float omw = 1.f - w;
    wp_pdl_enter();
    const FzStream in{&mv, &mf, sm.ring, sm.bars, z0 - 3, z1 + 2, x0, y0, !ZERO};
    if (tid == 0) {
        for (int s = 0; s < SLOTS; ++s) wptc::mbar_init(wptc::smem_u32(&sm.bars[s]), 1);
        wptc::mbar_init_fence();
        for (int p = in.pb; p < in.pb + SLOTS && p <= in.pe; ++p) in.issue(p);
    }
    const int tb = z0 - 3;  // plane table: planes z0 - 3 .. z1 + 2
    fz_tables(L, x0, y0, sm.gxs, sm.gys, sm.pz, tb, z1 - z0 + 6, tuni, ntiles, tile, fast_ok, tid);
    __syncthreads();
    int issued = min(in.pb + SLOTS - 1, in.pe);
    const FzCol c = fz_column(L, x0, y0, sm.gxs, sm.gys, w, tid);
    float* const dcol = dst + c.yq + (long)c.x * ny;
    float* const fcol = fc + (c.yq >> 1) + (long)(c.x >> 1) * ncy;
    float wxy[4] = {0.f, 0.f, 0.f, 0.f};
    if (tin) {
        const int xe = c.x & ~1;
        const double sx = L.d[0][xe] + L.d[0][xe + 1];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int y = c.yq + k, yb = y & ~1;
            const double sy = L.d[1][yb] + L.d[1][yb + 1];
            wxy[k] = (float)(L.d[1][y] / sy * (L.d[0][c.x] / sx));
        }
    }
    const Q4<float> z4 = zero4<float>();
    // histories: iterate at A-1; stage-1 values at A-2, A-1; stage-2 values at A-3, A-2; f at A-2, A-1
    Q4<float> v0m = z4, v1mm = z4, v1m = z4, v2mm = z4, v2m = z4, fm2 = z4, fm1 = z4;
    bool ok = in.wait(in.pb, err);
    int waited = in.pb;
    if (!ZERO && c.r1) v0m = ld4(in.slot(in.pb) + c.ov);
    for (int A = z0 - 2; A <= z1; A += 2) {
        ok = ok && in.wait(A, err) && in.wait(A + 1, err) && in.wait(A + 2, err);
        if (ok) waited = A + 2;
        const float* va = in.slot(A);
        const float* vb = in.slot(A + 1);
        const FzPlane Pa = sm.pz[A - tb], Pb = sm.pz[A + 1 - tb], Pm = sm.pz[A - 1 - tb], P2 = sm.pz[A - 2 - tb];
        // ---- stage 1: first sweep at planes A, A + 1
        Q4<float> v1a = z4, v1b = z4, ca = z4, cb = z4;
        const Q4<float> fa = c.r1 ? ld4(va + VPL + c.o) : z4, fb = c.r1 ? ld4(vb + VPL + c.o) : z4;
        if (!ZERO && c.r1) {
            ca = ld4(va + c.ov);
            cb = ld4(vb + c.ov);
        }
        if (tin && fz_fast(Pa) && fz_fast(Pb)) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if constexpr (ZERO) {
                    v1a.a[k] = c.wdstd[k] * fa.a[k];
                    v1b.a[k] = c.wdstd[k] * fb.a[k];
                }
            }
            if constexpr (!ZERO) {
                const FzNb na = fz_nb_in(va, c.ov), nb = fz_nb_in(vb, c.ov);
                v1a = fz_sweep_fast(c, Pa, ca, na.ym, na.yp, na.xm, na.xp, v0m, cb, fa, omw);
                v1b = fz_sweep_fast(c, Pb, cb, nb.ym, nb.yp, nb.xm, nb.xp, ca, ld4(in.slot(A + 2) + c.ov), fb, omw);
            }
        } else if (c.cin) {
            if constexpr (ZERO) {
                v1a = fz_sweep0(L, c, A, Pa, fa, w);
                v1b = fz_sweep0(L, c, A + 1, Pb, fb, w);
            } else {
                const FzNb na = fz_nb(va, c.ov, c.q), nb = fz_nb(vb, c.ov, c.q);
                v1a = fz_sweep(L, c, A, Pa, ca, na.ym, na.yp, na.xm, na.xp, v0m, cb, fa, w);
                v1b = fz_sweep(L, c, A + 1, Pb, cb, nb.ym, nb.yp, nb.xm, nb.xp, ca, ld4(in.slot(A + 2) + c.ov), fb, w);
            }
        }
        v0m = cb;
        if (c.r1) {
            st4(fz_stage(sm.b1, A) + c.o, v1a);
            st4(fz_stage(sm.b1, A + 1) + c.o, v1b);
        }
        ok = __syncthreads_and(ok);
        if (!ok) break;
        // planes up to A + 1 are consumed (A + 1's centre is in v0m): refill their slots
        {
            const int upto = min(A + 1 + SLOTS, in.pe);
            if (tid == 0)
                for (int p = issued + 1; p <= upto; ++p) in.issue(p);
            issued = max(issued, upto);
        }
        // ---- stage 2: second sweep at planes A - 1, A
        Q4<float> v2a = z4, v2b = z4;
        if (tin) {
            const FzNb nm = fz_nb_in(fz_stage(sm.b1, A - 1), c.o), na = fz_nb_in(fz_stage(sm.b1, A), c.o);
            if (fz_fast(Pm) && fz_fast(Pa)) {
                v2a = fz_sweep_fast(c, Pm, v1m, nm.ym, nm.yp, nm.xm, nm.xp, v1mm, v1a, fm1, omw);
                v2b = fz_sweep_fast(c, Pa, v1a, na.ym, na.yp, na.xm, na.xp, v1m, v1b, fa, omw);
            } else {
                v2a = fz_sweep(L, c, A - 1, Pm, v1m, nm.ym, nm.yp, nm.xm, nm.xp, v1mm, v1a, fm1, w);
                v2b = fz_sweep(L, c, A, Pa, v1a, na.ym, na.yp, na.xm, na.xp, v1m, v1b, fa, w);
            }
            if (A - 1 >= z0 && A - 1 < z1) st4(dcol + (long)(A - 1) * sxy, v2a);
            if (A >= z0 && A < z1) st4(dcol + (long)A * sxy, v2b);
        } else if (c.r2 && c.cin) {
            const FzNb nm = fz_nb(fz_stage(sm.b1, A - 1), c.o, c.q), na = fz_nb(fz_stage(sm.b1, A), c.o, c.q);
            v2a = fz_sweep(L, c, A - 1, Pm, v1m, nm.ym, nm.yp, nm.xm, nm.xp, v1mm, v1a, fm1, w);
            v2b = fz_sweep(L, c, A, Pa, v1a, na.ym, na.yp, na.xm, na.xp, v1m, v1b, fa, w);
        }
        if (c.r2) {
            st4(fz_stage(sm.b2, A - 1) + c.o, v2a);
            st4(fz_stage(sm.b2, A) + c.o, v2b);
        }
        __syncthreads();
        // ---- stage 3: residual at planes A - 2, A - 1 (one coarse plane), restricted
        if (tin && A - 2 >= z0) {
            const FzNb n2 = fz_nb_in(fz_stage(sm.b2, A - 2), c.o), n1 = fz_nb_in(fz_stage(sm.b2, A - 1), c.o);
            Q4<float> r2, r1;
            if (fz_fast(P2) && fz_fast(Pm)) {
                r2 = fz_resid_fast(c, P2, v2m, n2.ym, n2.yp, n2.xm, n2.xp, v2mm, v2a, fm2);
                r1 = fz_resid_fast(c, Pm, v2a, n1.ym, n1.yp, n1.xm, n1.xp, v2m, v2b, fm1);
            } else {
                r2 = fz_resid(L, c, A - 2, P2, v2m, n2.ym, n2.yp, n2.xm, n2.xp, v2mm, v2a, fm2);
                r1 = fz_resid(L, c, A - 1, Pm, v2a, n1.ym, n1.yp, n1.xm, n1.xp, v2m, v2b, fm1);
            }
            Q4<float> acc = z4;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                acc.a[k] += P2.wz * wxy[k] * r2.a[k];
                acc.a[k] += Pm.wz * wxy[k] * r1.a[k];
            }
            const float ya = acc.a[0] + acc.a[1], yb = acc.a[2] + acc.a[3];
            // lanes l and l + 8 hold the x pair (x even, x + 1) of the same coarse cells
            const float oa = __shfl_down_sync(0xffffffffu, ya, TY / 4);
            const float ob = __shfl_down_sync(0xffffffffu, yb, TY / 4);
            if (!(c.x & 1)) {
                float* o = fcol + (long)((A - 2) >> 1) * csxy;
                o[0] = ya + oa;
                o[1] = yb + ob;
            }
        }
        v1mm = v1a;
        v1m = v1b;
        v2mm = v2a;
        v2m = v2b;
        fm2 = fa;
        fm1 = fb;
    }
    if (!ok && tid == 0) {
        // a wait gave up: let the copies still in flight land before the CTA's shared memory goes
        for (int p = waited + 1; p <= issued; ++p) in.wait(p, err);
    }
}

// Prolongation + post-smoothing.  ACC: the result is added to the FP64 iterate p64 (the refinement
// update) instead of being stored into dst.  Two planes per iteration as cycle_down_kernel: stage 1
// (iterate + prolonged correction) at A, A+1, stage 2 (first sweep) at A-1, A, stage 3 (second
// sweep, stored) at A-2, A-1.
template <bool ACC>
__global__ void __launch_bounds__(fz::THREADS, 1)
    cycle_up_kernel(const __grid_constant__ CUtensorMap mv, const __grid_constant__ CUtensorMap mf,
                    float* __restrict__ dst, double* __restrict__ p64, const float* __restrict__ vc, Lvl<float> L,
                    const unsigned char* __restrict__ tuni, float w, int zc, int fast_ok, int* __restrict__ err) {
    using namespace fz;
    extern __shared__ __align__(128) float fz_raw[];
    const FzSmem sm = fz_smem(fz_raw);
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const int nty = ny / TY, ntiles = nty * (nx / TX);
    const int tile = blockIdx.x, x0 = (tile / nty) * TX, y0 = (tile - (tile / nty) * nty) * TY;
    const int z0 = blockIdx.y * zc, z1 = min(z0 + zc, nz);
    const int tid = threadIdx.x;
    const bool tin = tid < NIN;
    const int ncx = nx >> 1, ncy = ny >> 1, ncz = nz >> 1;
    const long sxy = (long)nx * ny;
    const float omw = 1.f - w;
    wp_pdl_enter();
    // stage 1 reads planes A and A + 1 only: the stream starts at the first stage-1 plane
    const FzStream in{&mv, &mf, sm.ring, sm.bars, z0 - 2, z1 + 1, x0, y0, true};
    if (tid == 0) {
        for (int s = 0; s < SLOTS; ++s) wptc::mbar_init(wptc::smem_u32(&sm.bars[s]), 1);
        wptc::mbar_init_fence();
        for (int p = in.pb; p < in.pb + SLOTS && p <= in.pe; ++p) in.issue(p);
    }
    const int tb = z0 - 3;  // plane table: planes z0 - 3 .. z1 + 2
    fz_tables(L, x0, y0, sm.gxs, sm.gys, sm.pz, tb, z1 - z0 + 6, tuni, ntiles, tile, fast_ok, tid);
    __syncthreads();
    int issued = min(in.pb + SLOTS - 1, in.pe);
    const FzCol c = fz_column(L, x0, y0, sm.gxs, sm.gys, w, tid);
    const long col = c.yq + (long)c.x * ny;
    const Q4<float> z4 = zero4<float>();
    const Q4<double> zd = zero4<double>();
    // histories: prolonged iterate at A-2, A-1; first-sweep values at A-3, A-2; f at A-2, A-1
    Q4<float> u1mm = z4, u1m = z4, s1mm = z4, s1m = z4, fm2 = z4, fm1 = z4;
    Q4<double> pa2 = zd, pa1 = zd;  // FP64 iterate of planes A-2, A-1 (loaded one iteration ahead)
    bool ok = true;
    int waited = in.pb - 1;
    for (int A = z0 - 2; A <= z1; A += 2) {
        ok = ok && in.wait(A, err) && in.wait(A + 1, err);
        if (ok) waited = A + 1;
        const float* va = in.slot(A);
        const float* vb = in.slot(A + 1);
        Q4<double> pn0 = zd, pn1 = zd;
        if (ACC && tin) {
            if (A >= z0 && A < z1) pn0 = ld4(p64 + col + (long)A * sxy);
            if (A + 1 >= z0 && A + 1 < z1) pn1 = ld4(p64 + col + (long)(A + 1) * sxy);
        }
        const FzPlane Pa = sm.pz[A - tb], Pb = sm.pz[A + 1 - tb], Pm = sm.pz[A - 1 - tb], P2 = sm.pz[A - 2 - tb];
        // ---- stage 1: iterate + prolonged coarse correction at planes A, A + 1
        Q4<float> ua = z4, ub = z4;
        const Q4<float> fa = c.r1 ? ld4(va + VPL + c.o) : z4, fb = c.r1 ? ld4(vb + VPL + c.o) : z4;
        if (c.cin && (Pa.mode & IN)) {  // A in the level implies A + 1 (nz even, A even)
            Q4<float> ia, ib;
            fz_prolong2(vc, c.x, c.yq, A, ncx, ncy, ncz, ia, ib);
            const Q4<float> xa = ld4(va + c.ov), xb = ld4(vb + c.ov);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                ua.a[k] = xa.a[k] + ia.a[k];
                ub.a[k] = xb.a[k] + ib.a[k];
            }
        }
        if (c.r1) {
            st4(fz_stage(sm.b1, A) + c.o, ua);
            st4(fz_stage(sm.b1, A + 1) + c.o, ub);
        }
        ok = __syncthreads_and(ok);
        if (!ok) break;
        // planes up to A + 1 are consumed: refill their slots
        {
            const int upto = min(A + 1 + SLOTS, in.pe);
            if (tid == 0)
                for (int p = issued + 1; p <= upto; ++p) in.issue(p);
            issued = max(issued, upto);
        }
        // ---- stage 2: first post-sweep at planes A - 1, A
        Q4<float> sa = z4, sb = z4;
        if (tin) {
            const FzNb nm = fz_nb_in(fz_stage(sm.b1, A - 1), c.o), na = fz_nb_in(fz_stage(sm.b1, A), c.o);
            if (fz_fast(Pm) && fz_fast(Pa)) {
                sa = fz_sweep_fast(c, Pm, u1m, nm.ym, nm.yp, nm.xm, nm.xp, u1mm, ua, fm1, omw);
                sb = fz_sweep_fast(c, Pa, ua, na.ym, na.yp, na.xm, na.xp, u1m, ub, fa, omw);
            } else {
                sa = fz_sweep(L, c, A - 1, Pm, u1m, nm.ym, nm.yp, nm.xm, nm.xp, u1mm, ua, fm1, w);
                sb = fz_sweep(L, c, A, Pa, ua, na.ym, na.yp, na.xm, na.xp, u1m, ub, fa, w);
            }
        } else if (c.r2 && c.cin) {
            const FzNb nm = fz_nb(fz_stage(sm.b1, A - 1), c.o, c.q), na = fz_nb(fz_stage(sm.b1, A), c.o, c.q);
            sa = fz_sweep(L, c, A - 1, Pm, u1m, nm.ym, nm.yp, nm.xm, nm.xp, u1mm, ua, fm1, w);
            sb = fz_sweep(L, c, A, Pa, ua, na.ym, na.yp, na.xm, na.xp, u1m, ub, fa, w);
        }
        if (c.r2) {
            st4(fz_stage(sm.b2, A - 1) + c.o, sa);
            st4(fz_stage(sm.b2, A) + c.o, sb);
        }
        __syncthreads();
        // ---- stage 3: second post-sweep at planes A - 2, A - 1, stored or added to the FP64 iterate
        if (tin && A - 2 >= z0) {
            const FzNb n2 = fz_nb_in(fz_stage(sm.b2, A - 2), c.o), n1 = fz_nb_in(fz_stage(sm.b2, A - 1), c.o);
            Q4<float> s2a, s2b;
            if (fz_fast(P2) && fz_fast(Pm)) {
                s2a = fz_sweep_fast(c, P2, s1m, n2.ym, n2.yp, n2.xm, n2.xp, s1mm, sa, fm2, omw);
                s2b = fz_sweep_fast(c, Pm, sa, n1.ym, n1.yp, n1.xm, n1.xp, s1m, sb, fm1, omw);
            } else {
                s2a = fz_sweep(L, c, A - 2, P2, s1m, n2.ym, n2.yp, n2.xm, n2.xp, s1mm, sa, fm2, w);
                s2b = fz_sweep(L, c, A - 1, Pm, sa, n1.ym, n1.yp, n1.xm, n1.xp, s1m, sb, fm1, w);
            }
            if constexpr (ACC) {
                Q4<double> qa = pa2, qb = pa1;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    qa.a[k] += (double)s2a.a[k];
                    qb.a[k] += (double)s2b.a[k];
                }
                st4(p64 + col + (long)(A - 2) * sxy, qa);
                st4(p64 + col + (long)(A - 1) * sxy, qb);
            } else {
                st4(dst + col + (long)(A - 2) * sxy, s2a);
                st4(dst + col + (long)(A - 1) * sxy, s2b);
            }
        }
        u1mm = ua;
        u1m = ub;
        s1mm = sa;
        s1m = sb;
        fm2 = fa;
        fm1 = fb;
        pa2 = pn0;
        pa1 = pn1;
    }
    if (!ok && tid == 0) {
        for (int p = waited + 1; p <= issued; ++p) in.wait(p, err);
    }
}

// Per (plane, tile) of a level: 1 when every interior face fraction of the first-stage region's
// cells (x0-2 .. x0+33, y0-4 .. y0+35, within the level) is exactly 1.  One CTA per (tile, plane).
__global__ void __launch_bounds__(256) tile_uni_kernel(unsigned char* __restrict__ tuni, Lvl<float> L) {
    const int nty = L.ny / fz::TY, tile = blockIdx.x, z = blockIdx.y;
    const int x0 = (tile / nty) * fz::TX, y0 = (tile - (tile / nty) * nty) * fz::TY;
    const long sxy = (long)L.nx * L.ny, sax = (long)(L.nx + 1) * L.ny;
    bool u = true;
    for (int j = threadIdx.x; j < fz::RX * fz::RY; j += blockDim.x) {
        const int x = x0 - 2 + j / fz::RY, y = y0 - 4 + j % fz::RY;
        if (x < 0 || x >= L.nx || y < 0 || y >= L.ny) continue;
        const long i = y + (long)x * L.ny + z * sxy, iax = y + (long)x * L.ny + z * sax;
        if (x > 0 && L.ax[iax] != 1.f) u = false;
        if (x + 1 < L.nx && L.ax[iax + L.ny] != 1.f) u = false;
        if (y > 0 && L.fyc[i] != 1.f) u = false;
        if (y + 1 < L.ny && L.fyc[i + 1] != 1.f) u = false;
        if (z > 0 && L.az[i] != 1.f) u = false;
        if (z + 1 < L.nz && L.az[i + sxy] != 1.f) u = false;
    }
    u = __syncthreads_and(u);
    if (threadIdx.x == 0) tuni[(long)z * gridDim.x + tile] = u ? 1 : 0;
}
