// wp_conv.cu -- 3x3x3 "same" convolutions of channels-last BF16 volumes on the tcgen05 tensor cores
// (FP32 accumulation in TMEM), the building block of the warm-start network.  No reference
// counterpart: the reference has no learned component.
//
// Layouts.  Activations: [z][x][y][c] BF16 (c fastest), c in {16, 32, 64}.  Weights of one input
// part: [tap][cout][cin] BF16 with tap = (dz * 3 + dx) * 3 + dy, offsets d - 1 (zero padding).
//
// Forward / input-gradient kernel (implicit GEMM, K-major operands).  A CTA owns a tile of
// M = 128 voxels of one z plane (yt consecutive y times xt consecutive x, yt * xt = 128) and all
// cout outputs.  K runs over (input part, tap, cin): per tap a TMA load brings the shifted
// [128 voxels][cin] block of the input (out-of-range voxels arrive as zeros = the padding) and the
// [cout][cin] weight block, each row one swizzle span (cin * 2 bytes = 32/64/128 B), which is the
// canonical K-major UMMA layout; cin / 16 tcgen05.mma (M=128, N=cout, K=16) accumulate into TMEM.
// Warp roles: warp 0 issues TMA, warp 1 owns TMEM and issues the MMAs, warps 2-5 drain TMEM
// (tcgen05.ld, one voxel per thread) and apply bias / skip-add / ReLU mask / ReLU, storing BF16.
// The input gradient of a convolution is the same kernel on the output gradient with the weights
// transposed and flipped ([26 - tap][cin][cout]).
//
// Weight-gradient kernel (MN-major operands).  dW[tap][co][ci] = sum_v dY[v][co] X[v + off(tap)][ci]
// is a GEMM with M = (tap, ci) rows, N = cout, K = voxels: a CTA owns 128 / cin taps (one M tile
// of 128 rows) and a range of voxel tiles; per voxel tile it TMA-loads the shifted input block of
// each of its taps (each an MN-major swizzle atom of width cin, stacked along M) and the output
// gradient block (MN-major, width cout), issues 8 MMAs of K = 16 voxels, and finally adds its
// partial [128][cout] tile into the FP32 weight gradient with atomics.
#include "wp_common.cuh"
#include "wp_tc.cuh"

#include <cstring>
#include <mutex>

using namespace wptc;

namespace {

constexpr int kThreads = 192;
constexpr int kStagesF = 4;
constexpr int kSlotA = 16384;  // 128 rows x 64 channels x 2 B
constexpr int kSlotB = 8192;   // 64 x 64 x 2 B
constexpr int kStagesW = 3;
constexpr int kSlotWA = 32768;  // 128 x 128 x 2 B
constexpr int kSlotWB = 16384;  // 128 x 64 x 2 B

__device__ __forceinline__ void store_bf16_row(__nv_bfloat16* dst, const float* v, int n) {
    for (int c = 0; c < n; c += 8) {
        __nv_bfloat162 h[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(v[c + 2 * k], v[c + 2 * k + 1]);
        *reinterpret_cast<uint4*>(dst + c) = *reinterpret_cast<uint4*>(h);
    }
}

__device__ __forceinline__ void load_bf16_row(const __nv_bfloat16* src, float* v, int n) {
    for (int c = 0; c < n; c += 8) {
        uint4 u = *reinterpret_cast<const uint4*>(src + c);
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 f = __bfloat1622float2(h[k]);
            v[c + 2 * k] = f.x;
            v[c + 2 * k + 1] = f.y;
        }
    }
}

struct TileGeo {
    int yt, xt, nty, ntx;
};

// After a pipeline wait gave up: waits (bounded) for the tile loads issued but never consumed, steps
// [consumed, issued) of the ring of full barriers, so that no copy into this CTA's shared memory is
// in flight when it exits.  The withheld step was never issued.
__device__ __forceinline__ void drain_copies(uint32_t bar_full, int stages, int consumed, int issued, int withheld,
                                             int* err) {
    for (int k = consumed; k < issued; ++k)
        if (k != withheld && !mbar_wait(bar_full + 8 * (k % stages), (k / stages) & 1, err)) return;
}

template <int COUT>
__global__ void __launch_bounds__(kThreads, 1)
    conv3_fwd_kernel(const __grid_constant__ CUtensorMap xm0, const __grid_constant__ CUtensorMap wm0,
                     const __grid_constant__ CUtensorMap xm1, const __grid_constant__ CUtensorMap wm1, int cin0,
                     int cin1, int nparts, __nv_bfloat16* __restrict__ out, const float* __restrict__ bias,
                     const __nv_bfloat16* __restrict__ addend, const __nv_bfloat16* __restrict__ mask, int relu, int nx,
                     int ny, int nz, TileGeo tg, int* err, int withhold, unsigned long long lim) {
    constexpr int NCOL = COUT < 32 ? 32 : COUT;
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* basep = smem_raw + (base - raw);
    const uint32_t bar_full = base + kStagesF * (kSlotA + kSlotB);
    const uint32_t bar_empty = bar_full + 8 * kStagesF;
    const uint32_t bar_acc = bar_empty + 8 * kStagesF;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(basep + kStagesF * (kSlotA + kSlotB) + 16 * kStagesF + 8);
    volatile int* s_consumed = reinterpret_cast<volatile int*>(tmem_slot + 1);
    volatile int* s_fail = reinterpret_cast<volatile int*>(tmem_slot + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (blockIdx.x != 0) withhold = -1;
    long t = blockIdx.x;
    const int ty = (int)(t % tg.nty);
    t /= tg.nty;
    const int tx = (int)(t % tg.ntx);
    const int z = (int)(t / tg.ntx);
    const int y0 = ty * tg.yt, x0 = tx * tg.xt;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStagesF; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, 1);
        }
        mbar_init(bar_acc, 1);
        mbar_init_fence();
    }
    if (warp == 1) {
        tmem_alloc(smem_u32(tmem_slot), NCOL);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int nk = 27 * nparts;

    int issued = 0;
    if (warp == 0 && lane == 0) {
        for (int k = 0; k < nk; ++k) {
            const int s = k % kStagesF;
            if (!mbar_wait(bar_empty + 8 * s, ((k / kStagesF) & 1) ^ 1, err, lim)) break;
            issued = k + 1;
            if (k == withhold) continue;
            const int part = k / 27, tap = k % 27;
            const int cin = part ? cin1 : cin0;
            const int dz = tap / 9, dx = (tap / 3) % 3, dy = tap % 3;
            const uint32_t a = base + s * (kSlotA + kSlotB), b = a + kSlotA;
            mbar_expect_tx(bar_full + 8 * s, (uint32_t)(128 * cin * 2 + COUT * cin * 2));
            tma_load_4d(a, part ? &xm1 : &xm0, bar_full + 8 * s, 0, y0 + dy - 1, x0 + dx - 1, z + dz - 1);
            tma_load_2d(b, part ? &wm1 : &wm0, bar_full + 8 * s, 0, tap * COUT);
        }
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = idesc_bf16_f32(128, COUT, 0, 0);
        int k = 0;
        for (; k < nk; ++k) {
            const int s = k % kStagesF;
            if (!mbar_wait(bar_full + 8 * s, (k / kStagesF) & 1, err, lim)) break;
            tc_fence_after();
            const int cin = (k / 27) ? cin1 : cin0;
            const uint32_t rowb = (uint32_t)cin * 2, lay = sw_code(cin * 2);
            const uint32_t a = base + s * (kSlotA + kSlotB), b = a + kSlotA;
            for (int j = 0; j < cin / 16; ++j) {
                const uint64_t ad = smem_desc(a + 32 * j, 16, 8 * rowb, lay);
                const uint64_t bd = smem_desc(b + 32 * j, 16, 8 * rowb, lay);
                umma_f16(tmem, ad, bd, idesc, (k | j) != 0);
            }
            umma_commit(bar_empty + 8 * s);
        }
        *s_consumed = k;
        *s_fail = k < nk;
        umma_commit(bar_acc);  // also on failure: bar_acc then tracks the MMAs already issued
    }
    bool ready = false;
    if (warp >= 2) ready = mbar_wait(bar_acc, 0, err);
    __syncthreads();
    if (warp == 0 && lane == 0) drain_copies(bar_full, kStagesF, *s_consumed, issued, withhold, err);
    if (warp >= 2) {
        const int q = warp & 3;
        const int m = q * 32 + lane;
        ready = ready && !*s_fail;
        __syncwarp();  // tcgen05.ld is warp-collective
        tc_fence_after();
        float acc[COUT];
#pragma unroll
        for (int c = 0; c < COUT; c += 16) tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + c, acc + c);
        tmem_wait_ld();
        const int xi = m / tg.yt, yi = m - xi * tg.yt;
        const int x = x0 + xi, y = y0 + yi;
        if (ready && x < nx && y < ny) {
            const long v = ((long)z * nx + x) * ny + y;
            if (bias)
#pragma unroll
                for (int c = 0; c < COUT; ++c) acc[c] += bias[c];
            if (addend) {
                float a2[COUT];
                load_bf16_row(addend + v * COUT, a2, COUT);
#pragma unroll
                for (int c = 0; c < COUT; ++c) acc[c] += a2[c];
            }
            if (mask) {
                float mk[COUT];
                load_bf16_row(mask + v * COUT, mk, COUT);
#pragma unroll
                for (int c = 0; c < COUT; ++c) acc[c] = mk[c] > 0.f ? acc[c] : 0.f;
            }
            if (relu)
#pragma unroll
                for (int c = 0; c < COUT; ++c) acc[c] = fmaxf(acc[c], 0.f);
            store_bf16_row(out + v * COUT, acc, COUT);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, NCOL);
    }
}

template <int COUT>
__global__ void __launch_bounds__(kThreads, 1)
    conv3_wgrad_kernel(const __grid_constant__ CUtensorMap xm, const __grid_constant__ CUtensorMap gm, int cin,
                       float* __restrict__ dw, int nx, int ny, int nz, TileGeo tg, long ntiles, int tiles_per_cta,
                       int* err, int withhold, unsigned long long lim) {
    constexpr int NCOL = COUT < 32 ? 32 : COUT;
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* basep = smem_raw + (base - raw);
    const uint32_t bar_full = base + kStagesW * (kSlotWA + kSlotWB);
    const uint32_t bar_empty = bar_full + 8 * kStagesW;
    const uint32_t bar_acc = bar_empty + 8 * kStagesW;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(basep + kStagesW * (kSlotWA + kSlotWB) + 16 * kStagesW + 8);
    volatile int* s_consumed = reinterpret_cast<volatile int*>(tmem_slot + 1);
    volatile int* s_fail = reinterpret_cast<volatile int*>(tmem_slot + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (blockIdx.x != 0 || blockIdx.y != 0) withhold = -1;
    const int tpg = 128 / cin;             // taps per CTA (one M tile of 128 rows)
    const int tap0 = blockIdx.x * tpg;
    const int ntap = min(tpg, 27 - tap0);
    const long k0 = (long)blockIdx.y * tiles_per_cta;
    const int nk = (int)min((long)tiles_per_cta, ntiles - k0);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStagesW; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, 1);
        }
        mbar_init(bar_acc, 1);
        mbar_init_fence();
    }
    if (warp == 1) {
        tmem_alloc(smem_u32(tmem_slot), NCOL);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    int issued = 0;
    if (warp == 0 && lane == 0) {
        for (int k = 0; k < nk; ++k) {
            const int s = k % kStagesW;
            if (!mbar_wait(bar_empty + 8 * s, ((k / kStagesW) & 1) ^ 1, err, lim)) break;
            issued = k + 1;
            if (k == withhold) continue;
            long t = k0 + k;
            const int ty = (int)(t % tg.nty);
            t /= tg.nty;
            const int tx = (int)(t % tg.ntx);
            const int z = (int)(t / tg.ntx);
            const int y0 = ty * tg.yt, x0 = tx * tg.xt;
            const uint32_t a = base + s * (kSlotWA + kSlotWB), b = a + kSlotWA;
            mbar_expect_tx(bar_full + 8 * s, (uint32_t)(ntap * 128 * cin * 2 + 128 * COUT * 2));
            for (int j = 0; j < ntap; ++j) {
                const int tap = tap0 + j;
                const int dz = tap / 9, dx = (tap / 3) % 3, dy = tap % 3;
                tma_load_4d(a + j * 128 * cin * 2, &xm, bar_full + 8 * s, 0, y0 + dy - 1, x0 + dx - 1, z + dz - 1);
            }
            tma_load_4d(b, &gm, bar_full + 8 * s, 0, y0, x0, z);
        }
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = idesc_bf16_f32(128, COUT, 1, 1);
        const uint32_t rowa = (uint32_t)cin * 2, laya = sw_code(cin * 2);
        constexpr uint32_t rowb = COUT * 2, layb = sw_code(COUT * 2);
        int k = 0;
        for (; k < nk; ++k) {
            const int s = k % kStagesW;
            if (!mbar_wait(bar_full + 8 * s, (k / kStagesW) & 1, err, lim)) break;
            tc_fence_after();
            const uint32_t a = base + s * (kSlotWA + kSlotWB), b = a + kSlotWA;
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) {
                const uint64_t ad = smem_desc(a + kk * 16 * rowa, 128 * rowa, 8 * rowa, laya);
                const uint64_t bd = smem_desc(b + kk * 16 * rowb, 128 * rowb, 8 * rowb, layb);
                umma_f16(tmem, ad, bd, idesc, (k | kk) != 0);
            }
            umma_commit(bar_empty + 8 * s);
        }
        *s_consumed = k;
        *s_fail = k < nk || nk <= 0;
        umma_commit(bar_acc);  // also on failure: bar_acc then tracks the MMAs already issued
    }
    bool ready = false;
    if (warp >= 2) ready = mbar_wait(bar_acc, 0, err);
    __syncthreads();
    if (warp == 0 && lane == 0) drain_copies(bar_full, kStagesW, *s_consumed, issued, withhold, err);
    if (warp >= 2) {
        const int q = warp & 3;
        const int m = q * 32 + lane;
        ready = ready && !*s_fail;
        __syncwarp();  // tcgen05.ld is warp-collective
        tc_fence_after();
        float acc[COUT];
#pragma unroll
        for (int c = 0; c < COUT; c += 16) tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + c, acc + c);
        tmem_wait_ld();
        const int j = m / cin, ci = m - j * cin;
        if (ready && j < ntap) {
            float* d = dw + (long)(tap0 + j) * COUT * cin + ci;
#pragma unroll
            for (int co = 0; co < COUT; ++co) atomicAdd(d + (long)co * cin, acc[co]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, NCOL);
    }
}

// ------------------------------------------------------------------------------ host side
using wptc::EncodeTiledFn;
EncodeTiledFn encode_fn() { return wptc::encode_tiled(); }

CUtensorMapSwizzle swz(int bytes) {
    return bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
}

// [z][x][y][c] volume, box (c, yt, xt, 1)
bool map_volume(CUtensorMap* m, const void* p, int c, int nx, int ny, int nz, int yt, int xt) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)ny, (cuuint64_t)nx, (cuuint64_t)nz};
    const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)c * 2 * ny, (cuuint64_t)c * 2 * ny * nx};
    const cuuint32_t box[4] = {(cuuint32_t)c, (cuuint32_t)yt, (cuuint32_t)xt, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(p), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, swz(c * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// [27 * cout][cin] weights, box (cin, cout)
bool map_weights(CUtensorMap* m, const void* p, int cin, int cout) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cin, (cuuint64_t)27 * cout};
    const cuuint64_t strides[1] = {(cuuint64_t)cin * 2};
    const cuuint32_t box[2] = {(cuuint32_t)cin, (cuuint32_t)cout};
    const cuuint32_t es[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(p), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, swz(cin * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool chan_ok(int c) { return c == 16 || c == 32 || c == 64; }
bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

TileGeo tile_geo(int nx, int ny) {
    TileGeo g;
    g.yt = ny < 128 ? ny : 128;
    g.xt = 128 / g.yt;
    g.nty = (ny + g.yt - 1) / g.yt;
    g.ntx = (nx + g.xt - 1) / g.xt;
    return g;
}

int* err_flag() {
    static int* d[64] = {nullptr};
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!d[dev] && cudaMalloc((void**)&d[dev], sizeof(int)) == cudaSuccess) cudaMemset(d[dev], 0, sizeof(int));
    return d[dev];
}

template <int COUT>
cudaError_t launch_fwd(const CUtensorMap& x0, const CUtensorMap& w0, const CUtensorMap& x1, const CUtensorMap& w1,
                       int cin0, int cin1, int nparts, __nv_bfloat16* out, const float* bias,
                       const __nv_bfloat16* addend, const __nv_bfloat16* mask, int relu, int nx, int ny, int nz,
                       TileGeo tg, int* err, cudaStream_t s) {
    const size_t smem = 1024 + kStagesF * (kSlotA + kSlotB) + 16 * kStagesF + 32;
    int wh = -1;
    unsigned long long lim = wptc::kWaitLimitNs;
    if (!wp_take_withhold(WP_WAIT_SITE_CONV_PIPELINE, s, &wh, &lim)) wh = -1;
    auto k = conv3_fwd_kernel<COUT>;
    cudaError_t e = wp_set_smem(k, smem);
    if (e != cudaSuccess) return e;
    const long tiles = (long)tg.nty * tg.ntx * nz;
    k<<<(unsigned)tiles, kThreads, smem, s>>>(x0, w0, x1, w1, cin0, cin1, nparts, out, bias, addend, mask, relu, nx, ny,
                                              nz, tg, err, wh, lim);
    return cudaGetLastError();
}

template <int COUT>
cudaError_t launch_wgrad(const CUtensorMap& xm, const CUtensorMap& gm, int cin, float* dw, int nx, int ny, int nz,
                         TileGeo tg, int* err, cudaStream_t s) {
    const size_t smem = 1024 + kStagesW * (kSlotWA + kSlotWB) + 16 * kStagesW + 32;
    int wh = -1;
    unsigned long long lim = wptc::kWaitLimitNs;
    if (!wp_take_withhold(WP_WAIT_SITE_CONV_PIPELINE, s, &wh, &lim)) wh = -1;
    auto k = conv3_wgrad_kernel<COUT>;
    cudaError_t e = wp_set_smem(k, smem);
    if (e != cudaSuccess) return e;
    const long ntiles = (long)tg.nty * tg.ntx * nz;
    const int groups = (27 + 128 / cin - 1) / (128 / cin);
    // about two CTAs per SM in total
    long chunks = (2L * wp_sm_count() + groups - 1) / groups;
    if (chunks > ntiles) chunks = ntiles;
    const int per = (int)((ntiles + chunks - 1) / chunks);
    chunks = (ntiles + per - 1) / per;
    k<<<dim3(groups, (unsigned)chunks), kThreads, smem, s>>>(xm, gm, cin, dw, nx, ny, nz, tg, ntiles, per, err, wh, lim);
    return cudaGetLastError();
}

}  // namespace

// Error flag of the tensor-core kernels on the current device (a bounded wait that gave up).
wp_status wp_conv_check_error(cudaStream_t s) {
    int* e = err_flag();
    if (!e) return WP_OK;
    int h = 0;
    WP_CUDA_TRY(cudaMemcpyAsync(&h, e, sizeof(int), cudaMemcpyDeviceToHost, s));
    WP_CUDA_TRY(cudaStreamSynchronize(s));
    if (h) {
        cudaMemsetAsync(e, 0, sizeof(int), s);
        wp_set_error_msg("tensor-core convolution: a pipeline wait gave up; the outputs of the call are invalid");
        return WP_ERR_DEVICE_WAIT;
    }
    return WP_OK;
}

// out = act(sum over parts conv(x_p, w_p) + bias + addend) [masked]; see the file comment.
wp_status wp_conv3_forward_impl(void* out, const void* x0, int cin0, const void* w0, const void* x1, int cin1,
                                const void* w1, const float* bias, int cout, int nx, int ny, int nz, int relu,
                                const void* addend, const void* mask, cudaStream_t s) {
    const int nparts = x1 ? 2 : 1;
    if (!out || !x0 || !w0 || !chan_ok(cin0) || (x1 && (!w1 || !chan_ok(cin1))) || !chan_ok(cout) || !pow2(nx) ||
        !pow2(ny) || nz < 1 || nz > 65535) {
        wp_set_error_msg("wp_conv3_forward: channels must be 16/32/64, nx and ny powers of two");
        return WP_ERR_INVALID_ARG;
    }
    const TileGeo tg = tile_geo(nx, ny);
    CUtensorMap mx0, mw0, mx1, mw1;
    if (!map_volume(&mx0, x0, cin0, nx, ny, nz, tg.yt, tg.xt) || !map_weights(&mw0, w0, cin0, cout)) {
        wp_set_error_msg("wp_conv3_forward: tensor map encoding failed");
        return WP_ERR_CUDA;
    }
    if (x1) {
        if (!map_volume(&mx1, x1, cin1, nx, ny, nz, tg.yt, tg.xt) || !map_weights(&mw1, w1, cin1, cout)) {
            wp_set_error_msg("wp_conv3_forward: tensor map encoding failed");
            return WP_ERR_CUDA;
        }
    } else {
        mx1 = mx0;
        mw1 = mw0;
        cin1 = cin0;
    }
    int* err = err_flag();
    if (!err) { wp_set_error_msg("wp_conv3_forward: error flag allocation failed"); return WP_ERR_CUDA; }
    auto o = static_cast<__nv_bfloat16*>(out);
    auto ad = static_cast<const __nv_bfloat16*>(addend);
    auto mk = static_cast<const __nv_bfloat16*>(mask);
    cudaError_t e;
    const int tok = wp_prof_start(s);
    switch (cout) {
        case 16: e = launch_fwd<16>(mx0, mw0, mx1, mw1, cin0, cin1, nparts, o, bias, ad, mk, relu, nx, ny, nz, tg, err, s); break;
        case 32: e = launch_fwd<32>(mx0, mw0, mx1, mw1, cin0, cin1, nparts, o, bias, ad, mk, relu, nx, ny, nz, tg, err, s); break;
        default: e = launch_fwd<64>(mx0, mw0, mx1, mw1, cin0, cin1, nparts, o, bias, ad, mk, relu, nx, ny, nz, tg, err, s); break;
    }
    const double flops = 2.0 * 27.0 * (cin0 + (x1 ? cin1 : 0)) * cout * (double)nx * ny * nz;
    wp_prof_stop(tok, "conv3_tc", flops, s);
    if (e != cudaSuccess) { wp_set_cuda_error(e, "conv3 forward", __FILE__, __LINE__); return WP_ERR_CUDA; }
    return WP_OK;
}

// dw[tap][cout][cin] += sum_v gy[v][co] x[v + off(tap)][ci] (FP32, caller zeroes dw)
wp_status wp_conv3_wgrad_impl(float* dw, const void* x, int cin, const void* gy, int cout, int nx, int ny, int nz,
                              cudaStream_t s) {
    if (!dw || !x || !gy || !chan_ok(cin) || !chan_ok(cout) || !pow2(nx) || !pow2(ny) || nz < 1 || nz > 65535) {
        wp_set_error_msg("wp_conv3_wgrad: channels must be 16/32/64, nx and ny powers of two");
        return WP_ERR_INVALID_ARG;
    }
    const TileGeo tg = tile_geo(nx, ny);
    CUtensorMap mx, mg;
    if (!map_volume(&mx, x, cin, nx, ny, nz, tg.yt, tg.xt) || !map_volume(&mg, gy, cout, nx, ny, nz, tg.yt, tg.xt)) {
        wp_set_error_msg("wp_conv3_wgrad: tensor map encoding failed");
        return WP_ERR_CUDA;
    }
    int* err = err_flag();
    if (!err) { wp_set_error_msg("wp_conv3_wgrad: error flag allocation failed"); return WP_ERR_CUDA; }
    cudaError_t e;
    const int tok = wp_prof_start(s);
    switch (cout) {
        case 16: e = launch_wgrad<16>(mx, mg, cin, dw, nx, ny, nz, tg, err, s); break;
        case 32: e = launch_wgrad<32>(mx, mg, cin, dw, nx, ny, nz, tg, err, s); break;
        default: e = launch_wgrad<64>(mx, mg, cin, dw, nx, ny, nz, tg, err, s); break;
    }
    wp_prof_stop(tok, "conv3_wgrad_tc", 2.0 * 27.0 * cin * cout * (double)nx * ny * nz, s);
    if (e != cudaSuccess) { wp_set_cuda_error(e, "conv3 wgrad", __FILE__, __LINE__); return WP_ERR_CUDA; }
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_conv3_forward(void* out, const void* x0, int cin0, const void* w0, const void* x1,
                                                 int cin1, const void* w1, const float* bias, int cout, int nx, int ny,
                                                 int nz, int relu, const void* addend, const void* mask, void* stream) {
    wp_status st = wp_conv3_forward_impl(out, x0, cin0, w0, x1, cin1, w1, bias, cout, nx, ny, nz, relu, addend, mask,
                                         (cudaStream_t)stream);
    if (st != WP_OK) return st;
    return wp_conv_check_error((cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_conv3_wgrad(float* dw, const void* x, int cin, const void* gy, int cout, int nx,
                                               int ny, int nz, void* stream) {
    wp_status st = wp_conv3_wgrad_impl(dw, x, cin, gy, cout, nx, ny, nz, (cudaStream_t)stream);
    if (st != WP_OK) return st;
    return wp_conv_check_error((cudaStream_t)stream);
}
