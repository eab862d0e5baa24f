// wp_unet.cu -- the warm-start network: a 3-level 3D U-Net (3x3x3 convolutions, 16/32/64 channels,
// ~0.35M parameters, BF16 weights and activations, FP32 accumulation) that maps the pressure
// right-hand side b and the solid level set to a multigrid starting guess, with its trainer
// (forward, backward, Adam) on the GPU.  No reference counterpart.
//
//   in (b / rms(b), clamp(sdf / 4h, -1, 1), 14 zero channels)            n^3 x 16
//   c1a 16->16, c1b 16->16 = s1 -> avg-pool                                n^3
//   c2a 16->32, c2b 32->32 = s2 -> avg-pool                                (n/2)^3
//   c3a 32->64, c3b 64->64 = e3 -> nearest upsample                        (n/4)^3
//   d2a [s2 | up(e3)] 96->32, d2b 32->32 = e2 -> nearest upsample          (n/2)^3
//   d1a [s1 | up(e2)] 48->16, d1b 16->16 = e1 -> 1x1 head 16->1 = p tscale / rms(b)
// Every 3x3x3 convolution is followed by ReLU.  Skip concatenations are two input parts of one
// convolution (wp_conv.cu).  The loss is the mean over fluid cells (sdf > 0) of the squared error
// after removing the mean error over those cells (a constant offset is free: the multigrid
// operator has the constant in its null space).
#include "wp_common.cuh"

#include <cuda_bf16.h>

#include <cmath>
#include <new>
#include <random>
#include <vector>

wp_status wp_conv3_forward_impl(void* out, const void* x0, int cin0, const void* w0, const void* x1, int cin1,
                                const void* w1, const float* bias, int cout, int nx, int ny, int nz, int relu,
                                const void* addend, const void* mask, cudaStream_t s);
wp_status wp_conv3_wgrad_impl(float* dw, const void* x, int cin, const void* gy, int cout, int nx, int ny, int nz,
                              cudaStream_t s);
wp_status wp_conv_check_error(cudaStream_t s);

namespace {

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ void ld8(const bf16* p, float* v) {
    uint4 u = *reinterpret_cast<const uint4*>(p);
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float2 f = __bfloat1622float2(h[k]);
        v[2 * k] = f.x;
        v[2 * k + 1] = f.y;
    }
}
__device__ __forceinline__ void st8(bf16* p, const float* v) {
    __nv_bfloat162 h[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
    *reinterpret_cast<uint4*>(p) = *reinterpret_cast<uint4*>(h);
}

__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
    return t;
}

// acc[0] += sum b^2 over all cells
__global__ void sumsq_kernel(const float* __restrict__ b, long n, double* __restrict__ acc) {
    __shared__ double red[8];
    double s = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double v = b[i];
        s += v * v;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) atomicAdd(acc, s);
}

// in16[v] = (b / rms, clamp(sdf / 4h), 0 x 14)
__global__ void pack_kernel(bf16* __restrict__ in16, const float* __restrict__ b, const float* __restrict__ sdf, long n,
                            const double* __restrict__ acc, float inv4h) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double ms = acc[0] / (double)n;
    const float inv = ms > 0.0 ? (float)(1.0 / sqrt(ms)) : 0.f;
    float v[16] = {0.f};
    v[0] = b[i] * inv;
    v[1] = fminf(fmaxf(sdf[i] * inv4h, -1.f), 1.f);
    st8(in16 + i * 16, v);
    st8(in16 + i * 16 + 8, v + 8);
}

// 2x2x2 average pooling; one thread per (coarse voxel, 8 channels)
__global__ void pool_kernel(bf16* __restrict__ out, const bf16* __restrict__ in, int C, int nx, int ny, int nz) {
    const int cx = nx / 2, cy = ny / 2, cz = nz / 2, g = C / 8;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= (long)cx * cy * cz * g) return;
    const int cg = (int)(t % g);
    const long vc = t / g;
    const int y = (int)(vc % cy), x = (int)((vc / cy) % cx), z = (int)(vc / ((long)cy * cx));
    float acc[8] = {0.f}, v[8];
    for (int k = 0; k < 8; ++k) {
        const long fv = ((long)(2 * z + (k >> 2)) * nx + 2 * x + ((k >> 1) & 1)) * ny + 2 * y + (k & 1);
        ld8(in + fv * C + cg * 8, v);
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] += v[j];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] *= 0.125f;
    st8(out + vc * C + cg * 8, acc);
}

// fine gradient = (g_coarse[parent] / 8 + addend) masked by mask > 0; one thread per (fine voxel, 8 ch)
__global__ void pool_bwd_kernel(bf16* __restrict__ gin, const bf16* __restrict__ gout, const bf16* __restrict__ addend,
                                const bf16* __restrict__ mask, int C, int nx, int ny, int nz) {
    const int g = C / 8;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= (long)nx * ny * nz * g) return;
    const int cg = (int)(t % g);
    const long v = t / g;
    const int y = (int)(v % ny), x = (int)((v / ny) % nx), z = (int)(v / ((long)ny * nx));
    const long pv = ((long)(z / 2) * (nx / 2) + x / 2) * (ny / 2) + y / 2;
    float a[8], b[8], m[8];
    ld8(gout + pv * C + cg * 8, a);
    if (addend) ld8(addend + v * C + cg * 8, b);
    else
        for (int j = 0; j < 8; ++j) b[j] = 0.f;
    ld8(mask + v * C + cg * 8, m);
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = m[j] > 0.f ? a[j] * 0.125f + b[j] : 0.f;
    st8(gin + v * C + cg * 8, a);
}

// nearest upsampling x2; one thread per (fine voxel, 8 ch)
__global__ void up_kernel(bf16* __restrict__ out, const bf16* __restrict__ in, int C, int nx, int ny, int nz) {
    const int g = C / 8;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= (long)nx * ny * nz * g) return;
    const int cg = (int)(t % g);
    const long v = t / g;
    const int y = (int)(v % ny), x = (int)((v / ny) % nx), z = (int)(v / ((long)ny * nx));
    const long pv = ((long)(z / 2) * (nx / 2) + x / 2) * (ny / 2) + y / 2;
    *reinterpret_cast<uint4*>(out + v * C + cg * 8) = *reinterpret_cast<const uint4*>(in + pv * C + cg * 8);
}

// coarse gradient = sum of the 8 fine children, masked by mask > 0 (coarse); nx.. are fine extents
__global__ void up_bwd_kernel(bf16* __restrict__ gc, const bf16* __restrict__ gf, const bf16* __restrict__ mask, int C,
                              int nx, int ny, int nz) {
    const int cx = nx / 2, cy = ny / 2, cz = nz / 2, g = C / 8;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= (long)cx * cy * cz * g) return;
    const int cg = (int)(t % g);
    const long vc = t / g;
    const int y = (int)(vc % cy), x = (int)((vc / cy) % cx), z = (int)(vc / ((long)cy * cx));
    float acc[8] = {0.f}, v[8], m[8];
    for (int k = 0; k < 8; ++k) {
        const long fv = ((long)(2 * z + (k >> 2)) * nx + 2 * x + ((k >> 1) & 1)) * ny + 2 * y + (k & 1);
        ld8(gf + fv * C + cg * 8, v);
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] += v[j];
    }
    ld8(mask + vc * C + cg * 8, m);
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = m[j] > 0.f ? acc[j] : 0.f;
    st8(gc + vc * C + cg * 8, acc);
}

// pred[v] = wh . e1[v] + bh; out (optional) = pred * rms(b) / tscale
__global__ void head_kernel(float* __restrict__ pred, float* __restrict__ out, const bf16* __restrict__ e1,
                            const float* __restrict__ wh, long n, const double* __restrict__ acc, double tscale) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v[16];
    ld8(e1 + i * 16, v);
    ld8(e1 + i * 16 + 8, v + 8);
    float s = wh[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) s += wh[c] * v[c];
    pred[i] = s;
    if (out) out[i] = (float)(s * sqrt(acc[0] / (double)n) / tscale);
}

// pass 1 of the loss: acc[1] += sum over fluid of (pred - t), acc[2] += fluid count;
// t = p tscale / rms(b)
__global__ void loss_mean_kernel(const float* __restrict__ pred, const float* __restrict__ p,
                                 const float* __restrict__ sdf, long n, double* __restrict__ acc, double tscale) {
    __shared__ double red[8];
    const double ms = acc[0] / (double)n;
    const double inv = ms > 0.0 ? tscale / sqrt(ms) : 0.0;
    double s = 0.0, c = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        if (sdf[i] > 0.f) {
            s += (double)pred[i] - (double)p[i] * inv;
            c += 1.0;
        }
    s = block_sum(s, red);
    c = block_sum(c, red);
    if (threadIdx.x == 0) {
        atomicAdd(acc + 1, s);
        atomicAdd(acc + 2, c);
    }
}

// pass 2: g = 2 (r - mean r) / count on fluid cells, acc[3] += (r - mean r)^2 / count
__global__ void loss_grad_kernel(float* __restrict__ g, const float* __restrict__ pred, const float* __restrict__ p,
                                 const float* __restrict__ sdf, long n, double* __restrict__ acc, double tscale) {
    __shared__ double red[8];
    const double ms = acc[0] / (double)n;
    const double inv = ms > 0.0 ? tscale / sqrt(ms) : 0.0;
    const double cnt = fmax(acc[2], 1.0), mu = acc[1] / cnt;
    double l = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double r = 0.0;
        if (sdf[i] > 0.f) r = (double)pred[i] - (double)p[i] * inv - mu;
        g[i] = (float)(2.0 * r / cnt);
        l += r * r / cnt;
    }
    l = block_sum(l, red);
    if (threadIdx.x == 0) atomicAdd(acc + 3, l);
}

// head backward: ge1 = g * wh * (e1 > 0); gwh[c] += sum g e1[c], gwh[16] += sum g
__global__ void head_bwd_kernel(bf16* __restrict__ ge1, float* __restrict__ gwh, const float* __restrict__ g,
                                const bf16* __restrict__ e1, const float* __restrict__ wh, long n) {
    __shared__ double red[8];
    float part[17] = {0.f};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        float v[16], o[16];
        ld8(e1 + i * 16, v);
        ld8(e1 + i * 16 + 8, v + 8);
        const float gi = g[i];
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            part[c] += gi * v[c];
            o[c] = v[c] > 0.f ? gi * wh[c] : 0.f;
        }
        part[16] += gi;
        st8(ge1 + i * 16, o);
        st8(ge1 + i * 16 + 8, o + 8);
    }
    for (int c = 0; c < 17; ++c) {
        const double t = block_sum((double)part[c], red);
        if (threadIdx.x == 0) atomicAdd(gwh + c, (float)t);
    }
}

// gb[c] += sum_v gy[v][c]; thread per (voxel, 8 ch) with a grid-stride loop
__global__ void bias_grad_kernel(float* __restrict__ gb, const bf16* __restrict__ gy, int C, long n) {
    __shared__ float red[64];
    for (int c = threadIdx.x; c < C; c += blockDim.x) red[c] = 0.f;
    __syncthreads();
    const int g = C / 8;
    float acc[8] = {0.f};
    int mycg = -1;
    const long stride = (long)gridDim.x * blockDim.x;
    // stride is a multiple of g (blockDim = 256, g in {2, 4, 8}) so each thread keeps one channel group
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n * g; t += stride) {
        mycg = (int)(t % g);
        float v[8];
        ld8(gy + (t / g) * C + mycg * 8, v);
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] += v[j];
    }
    if (mycg >= 0)
        for (int j = 0; j < 8; ++j) atomicAdd(&red[mycg * 8 + j], acc[j]);
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(gb + c, red[c]);
}

// Adam (bias-corrected) on FP32 master weights
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long n, float lr, float b1, float b2, float eps, float c1, float c2) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// BF16 copies of a conv weight [27][cout][cin]: forward layout and input-gradient layout
// wt[26 - tap][ci][co] = w[tap][co][ci]
__global__ void weight_copies_kernel(bf16* __restrict__ w16, bf16* __restrict__ wt16, const float* __restrict__ w,
                                     int cout, int cin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 27 * cout * cin) return;
    const int t = i / (cout * cin), co = (i / cin) % cout, ci = i % cin;
    const bf16 h = __float2bfloat16_rn(w[i]);
    w16[i] = h;
    wt16[((26 - t) * cin + ci) * cout + co] = h;
}

struct Conv {
    int nparts = 1, cin[2] = {0, 0}, cout = 0;
    float* w[2] = {nullptr, nullptr};  // FP32 masters [27][cout][cin_p]
    float* gw[2] = {nullptr, nullptr};
    float* mw[2] = {nullptr, nullptr};
    float* vw[2] = {nullptr, nullptr};
    bf16* w16[2] = {nullptr, nullptr};
    bf16* wt16[2] = {nullptr, nullptr};
    float *b = nullptr, *gb = nullptr, *mb = nullptr, *vb = nullptr;
    long wsize(int p) const { return 27L * cout * cin[p]; }
};

}  // namespace

struct wp_unet {
    int n[3];            // finest extents (nx, ny, nz)
    Conv c[10];          // c1a c1b c2a c2b c3a c3b d2a d2b d1a d1b
    float *wh, *gwh, *mwh, *vwh;  // head [16 weights | bias]
    double* acc;         // [sum b^2, sum r, fluid count, loss]
    // activations (BF16 channels-last) and gradients
    bf16 *in16, *a1, *s1, *p1, *a2, *s2, *p2, *a3, *e3, *u2, *a4, *e2, *u1, *a5, *e1;
    bf16 *g_e1, *g_a5, *g_s1p, *g_u1, *g_e2, *g_a4, *g_s2p, *g_u2, *g_e3, *g_a3, *g_p2, *g_s2, *g_a2, *g_p1, *g_s1, *g_a1;
    float *pred, *gpred;
    int step;
    std::vector<void*> allocs;
};

namespace {

enum { C1A, C1B, C2A, C2B, C3A, C3B, D2A, D2B, D1A, D1B };

template <typename T>
cudaError_t alloc(wp_unet* h, T** p, size_t count) {
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
    if (e == cudaSuccess) h->allocs.push_back(*p);
    return e;
}

unsigned blocks(long n, int per = 256) { return (unsigned)((n + per - 1) / per); }

wp_status refresh_copies(wp_unet* h, cudaStream_t s) {
    for (auto& C : h->c)
        for (int p = 0; p < C.nparts; ++p)
            WP_KERNEL("unet_weights", 6.0 * C.wsize(p), s,
                      weight_copies_kernel<<<blocks(C.wsize(p)), 256, 0, s>>>(C.w16[p], C.wt16[p], C.w[p], C.cout,
                                                                              C.cin[p]));
    return WP_OK;
}

// the network works on p * tscale / rms(b): tscale = 4 pi^2 / Lx^2 (Lx = nx h, the domain length
// along x) makes the normalized pressure of a smooth right-hand side O(1)
double target_scale(const wp_unet* h, double hcell) {
    const double lx = h->n[0] * hcell;
    return 4.0 * M_PI * M_PI / (lx * lx);
}

long vox(const wp_unet* h, int level) {
    return (long)(h->n[0] >> level) * (h->n[1] >> level) * (h->n[2] >> level);
}

wp_status conv_fwd(wp_unet* h, int id, const bf16* x0, const bf16* x1, bf16* out, int level, cudaStream_t s) {
    const Conv& C = h->c[id];
    return wp_conv3_forward_impl(out, x0, C.cin[0], C.w16[0], x1, C.cin[1], x1 ? C.w16[1] : nullptr, C.b, C.cout,
                                 h->n[0] >> level, h->n[1] >> level, h->n[2] >> level, 1, nullptr, nullptr, s);
}

// input gradient of part p of conv id: out = conv(gy, wt_p) [masked]
wp_status conv_dgrad(wp_unet* h, int id, int p, const bf16* gy, bf16* out, const bf16* mask, int level, cudaStream_t s) {
    const Conv& C = h->c[id];
    return wp_conv3_forward_impl(out, gy, C.cout, C.wt16[p], nullptr, 0, nullptr, nullptr, C.cin[p], h->n[0] >> level,
                                 h->n[1] >> level, h->n[2] >> level, 0, nullptr, mask, s);
}

wp_status conv_wgrad(wp_unet* h, int id, int p, const bf16* x, const bf16* gy, int level, cudaStream_t s) {
    const Conv& C = h->c[id];
    wp_status st = wp_conv3_wgrad_impl(C.gw[p], x, C.cin[p], gy, C.cout, h->n[0] >> level, h->n[1] >> level,
                                       h->n[2] >> level, s);
    if (st != WP_OK || p != 0) return st;
    const long n = vox(h, level);
    WP_KERNEL("unet_bias_grad", 2.0 * n * C.cout, s,
              bias_grad_kernel<<<std::min<unsigned>(blocks(n * (C.cout / 8)), 4 * wp_sm_count()), 256, 0, s>>>(
                  C.gb, gy, C.cout, n));
    return WP_OK;
}

wp_status forward(wp_unet* h, const float* b, const float* sdf, double hcell, float* out, cudaStream_t s) {
    const long n0 = vox(h, 0), n1 = vox(h, 1), n2 = vox(h, 2);
    const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
    wp_status st;
    WP_CUDA_TRY(cudaMemsetAsync(h->acc, 0, 4 * sizeof(double), s));
    WP_KERNEL("unet_sumsq", 4.0 * n0, s,
              sumsq_kernel<<<std::min<unsigned>(blocks(n0), 4 * wp_sm_count()), 256, 0, s>>>(b, n0, h->acc));
    WP_KERNEL("unet_pack", 40.0 * n0, s,
              pack_kernel<<<blocks(n0), 256, 0, s>>>(h->in16, b, sdf, n0, h->acc, (float)(1.0 / (4.0 * hcell))));
    if ((st = conv_fwd(h, C1A, h->in16, nullptr, h->a1, 0, s)) != WP_OK) return st;
    if ((st = conv_fwd(h, C1B, h->a1, nullptr, h->s1, 0, s)) != WP_OK) return st;
    WP_KERNEL("unet_pool", 2.0 * 16 * (n0 + n1), s,
              pool_kernel<<<blocks(n1 * 2), 256, 0, s>>>(h->p1, h->s1, 16, nx, ny, nz));
    if ((st = conv_fwd(h, C2A, h->p1, nullptr, h->a2, 1, s)) != WP_OK) return st;
    if ((st = conv_fwd(h, C2B, h->a2, nullptr, h->s2, 1, s)) != WP_OK) return st;
    WP_KERNEL("unet_pool", 2.0 * 32 * (n1 + n2), s,
              pool_kernel<<<blocks(n2 * 4), 256, 0, s>>>(h->p2, h->s2, 32, nx >> 1, ny >> 1, nz >> 1));
    if ((st = conv_fwd(h, C3A, h->p2, nullptr, h->a3, 2, s)) != WP_OK) return st;
    if ((st = conv_fwd(h, C3B, h->a3, nullptr, h->e3, 2, s)) != WP_OK) return st;
    WP_KERNEL("unet_up", 2.0 * 64 * (n1 + n2), s,
              up_kernel<<<blocks(n1 * 8), 256, 0, s>>>(h->u2, h->e3, 64, nx >> 1, ny >> 1, nz >> 1));
    if ((st = conv_fwd(h, D2A, h->s2, h->u2, h->a4, 1, s)) != WP_OK) return st;
    if ((st = conv_fwd(h, D2B, h->a4, nullptr, h->e2, 1, s)) != WP_OK) return st;
    WP_KERNEL("unet_up", 2.0 * 32 * (n0 + n1), s,
              up_kernel<<<blocks(n0 * 4), 256, 0, s>>>(h->u1, h->e2, 32, nx, ny, nz));
    if ((st = conv_fwd(h, D1A, h->s1, h->u1, h->a5, 0, s)) != WP_OK) return st;
    if ((st = conv_fwd(h, D1B, h->a5, nullptr, h->e1, 0, s)) != WP_OK) return st;
    WP_KERNEL("unet_head", 40.0 * n0, s, head_kernel<<<blocks(n0), 256, 0, s>>>(h->pred, out, h->e1, h->wh, n0, h->acc,
                                                                     target_scale(h, hcell)));
    return WP_OK;
}

wp_status backward(wp_unet* h, const float* sdf, const float* p, double hcell, cudaStream_t s) {
    const long n0 = vox(h, 0);
    const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
    wp_status st;
    const unsigned rb = std::min<unsigned>(blocks(n0), 4 * wp_sm_count());
    WP_KERNEL("unet_loss", 12.0 * n0, s, loss_mean_kernel<<<rb, 256, 0, s>>>(h->pred, p, sdf, n0, h->acc, target_scale(h, hcell)));
    WP_KERNEL("unet_loss", 16.0 * n0, s, loss_grad_kernel<<<rb, 256, 0, s>>>(h->gpred, h->pred, p, sdf, n0, h->acc,
                                                                                   target_scale(h, hcell)));
    // zero the gradient accumulators
    for (auto& C : h->c) {
        for (int q = 0; q < C.nparts; ++q) WP_CUDA_TRY(cudaMemsetAsync(C.gw[q], 0, sizeof(float) * C.wsize(q), s));
        WP_CUDA_TRY(cudaMemsetAsync(C.gb, 0, sizeof(float) * C.cout, s));
    }
    WP_CUDA_TRY(cudaMemsetAsync(h->gwh, 0, sizeof(float) * 17, s));
    WP_KERNEL("unet_head_bwd", 40.0 * n0, s, head_bwd_kernel<<<rb, 256, 0, s>>>(h->g_e1, h->gwh, h->gpred, h->e1, h->wh, n0));
    // decoder level 1
    if ((st = conv_dgrad(h, D1B, 0, h->g_e1, h->g_a5, h->a5, 0, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, D1B, 0, h->a5, h->g_e1, 0, s)) != WP_OK) return st;
    if ((st = conv_dgrad(h, D1A, 0, h->g_a5, h->g_s1p, nullptr, 0, s)) != WP_OK) return st;
    if ((st = conv_dgrad(h, D1A, 1, h->g_a5, h->g_u1, nullptr, 0, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, D1A, 0, h->s1, h->g_a5, 0, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, D1A, 1, h->u1, h->g_a5, 0, s)) != WP_OK) return st;
    const long n1 = vox(h, 1), n2 = vox(h, 2);
    WP_KERNEL("unet_up_bwd", 2.0 * 32 * (n0 + n1), s,
              up_bwd_kernel<<<blocks(n1 * 4), 256, 0, s>>>(h->g_e2, h->g_u1, h->e2, 32, nx, ny, nz));
    // decoder level 2
    if ((st = conv_dgrad(h, D2B, 0, h->g_e2, h->g_a4, h->a4, 1, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, D2B, 0, h->a4, h->g_e2, 1, s)) != WP_OK) return st;
    if ((st = conv_dgrad(h, D2A, 0, h->g_a4, h->g_s2p, nullptr, 1, s)) != WP_OK) return st;
    if ((st = conv_dgrad(h, D2A, 1, h->g_a4, h->g_u2, nullptr, 1, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, D2A, 0, h->s2, h->g_a4, 1, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, D2A, 1, h->u2, h->g_a4, 1, s)) != WP_OK) return st;
    WP_KERNEL("unet_up_bwd", 2.0 * 64 * (n1 + n2), s,
              up_bwd_kernel<<<blocks(n2 * 8), 256, 0, s>>>(h->g_e3, h->g_u2, h->e3, 64, nx >> 1, ny >> 1, nz >> 1));
    // bottom
    if ((st = conv_dgrad(h, C3B, 0, h->g_e3, h->g_a3, h->a3, 2, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, C3B, 0, h->a3, h->g_e3, 2, s)) != WP_OK) return st;
    if ((st = conv_dgrad(h, C3A, 0, h->g_a3, h->g_p2, nullptr, 2, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, C3A, 0, h->p2, h->g_a3, 2, s)) != WP_OK) return st;
    WP_KERNEL("unet_pool_bwd", 2.0 * 32 * (n1 + n2) + 4.0 * 32 * n1, s,
              pool_bwd_kernel<<<blocks(n1 * 4), 256, 0, s>>>(h->g_s2, h->g_p2, h->g_s2p, h->s2, 32, nx >> 1, ny >> 1,
                                                             nz >> 1));
    // encoder level 2
    if ((st = conv_dgrad(h, C2B, 0, h->g_s2, h->g_a2, h->a2, 1, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, C2B, 0, h->a2, h->g_s2, 1, s)) != WP_OK) return st;
    if ((st = conv_dgrad(h, C2A, 0, h->g_a2, h->g_p1, nullptr, 1, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, C2A, 0, h->p1, h->g_a2, 1, s)) != WP_OK) return st;
    WP_KERNEL("unet_pool_bwd", 2.0 * 16 * (n0 + n1) + 4.0 * 16 * n0, s,
              pool_bwd_kernel<<<blocks(n0 * 2), 256, 0, s>>>(h->g_s1, h->g_p1, h->g_s1p, h->s1, 16, nx, ny, nz));
    // encoder level 1
    if ((st = conv_dgrad(h, C1B, 0, h->g_s1, h->g_a1, h->a1, 0, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, C1B, 0, h->a1, h->g_s1, 0, s)) != WP_OK) return st;
    if ((st = conv_wgrad(h, C1A, 0, h->in16, h->g_a1, 0, s)) != WP_OK) return st;
    return WP_OK;
}

wp_status adam(wp_unet* h, double lr, cudaStream_t s) {
    h->step += 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - powf(b1, (float)h->step), c2 = 1.f - powf(b2, (float)h->step);
    auto upd = [&](float* w, float* g, float* m, float* v, long n) {
        adam_kernel<<<blocks(n), 256, 0, s>>>(w, g, m, v, n, (float)lr, b1, b2, eps, c1, c2);
    };
    for (auto& C : h->c) {
        for (int p = 0; p < C.nparts; ++p) WP_KERNEL("unet_adam", 20.0 * C.wsize(p), s, upd(C.w[p], C.gw[p], C.mw[p], C.vw[p], C.wsize(p)));
        WP_KERNEL("unet_adam", 20.0 * C.cout, s, upd(C.b, C.gb, C.mb, C.vb, C.cout));
    }
    WP_KERNEL("unet_adam", 20.0 * 17, s, upd(h->wh, h->gwh, h->mwh, h->vwh, 17));
    return refresh_copies(h, s);
}

// visits every parameter tensor (FP32 masters and the head) in a fixed order
template <typename F>
void each_param(wp_unet* h, F&& f) {
    for (auto& C : h->c) {
        for (int p = 0; p < C.nparts; ++p) f(C.w[p], C.gw[p], C.wsize(p));
        f(C.b, C.gb, (long)C.cout);
    }
    f(h->wh, h->gwh, 17L);
}

}  // namespace

extern "C" CUWHHD_API wp_status wp_unet_create(wp_unet** out, int nx, int ny, int nz, unsigned long long seed) {
    if (!out) { wp_set_error_msg("wp_unet_create: null handle"); return WP_ERR_INVALID_ARG; }
    *out = nullptr;
    auto p2 = [](int v) { return v >= 16 && (v & (v - 1)) == 0; };
    if (!p2(nx) || !p2(ny) || nz < 4 || nz % 4 != 0 || nz > 4096) {
        wp_set_error_msg("wp_unet_create: nx, ny must be powers of two >= 16 and nz a multiple of 4");
        return WP_ERR_INVALID_ARG;
    }
    wp_unet* h = new (std::nothrow) wp_unet();
    if (!h) return WP_ERR_INVALID_ARG;
    h->n[0] = nx;
    h->n[1] = ny;
    h->n[2] = nz;
    const int spec[10][3] = {{16, 0, 16}, {16, 0, 16}, {16, 0, 32}, {32, 0, 32}, {32, 0, 64},
                             {64, 0, 64}, {32, 64, 32}, {32, 0, 32}, {16, 32, 16}, {16, 0, 16}};
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 10 && e == cudaSuccess; ++i) {
        Conv& C = h->c[i];
        C.cin[0] = spec[i][0];
        C.cin[1] = spec[i][1];
        C.nparts = spec[i][1] ? 2 : 1;
        C.cout = spec[i][2];
        const int fan_in = 27 * (C.cin[0] + C.cin[1]);
        const float sd = std::sqrt(2.f / (float)fan_in);
        for (int p = 0; p < C.nparts && e == cudaSuccess; ++p) {
            const long n = C.wsize(p);
            std::vector<float> w(n);
            // the first layer sees 2 live input channels out of 16
            const float sdp = (i == C1A) ? std::sqrt(2.f / (27.f * 2.f)) : sd;
            for (auto& v : w) v = nd(rng) * sdp;
            if (i == C1A)
                for (long k = 0; k < n; ++k)
                    if (k % C.cin[0] >= 2) w[k] = 0.f;
            if ((e = alloc(h, &C.w[p], n)) != cudaSuccess) break;
            if ((e = alloc(h, &C.gw[p], n)) != cudaSuccess) break;
            if ((e = alloc(h, &C.mw[p], n)) != cudaSuccess) break;
            if ((e = alloc(h, &C.vw[p], n)) != cudaSuccess) break;
            if ((e = alloc(h, &C.w16[p], n)) != cudaSuccess) break;
            if ((e = alloc(h, &C.wt16[p], n)) != cudaSuccess) break;
            e = cudaMemcpy(C.w[p], w.data(), sizeof(float) * n, cudaMemcpyHostToDevice);
            if (e == cudaSuccess) e = cudaMemset(C.mw[p], 0, sizeof(float) * n);
            if (e == cudaSuccess) e = cudaMemset(C.vw[p], 0, sizeof(float) * n);
        }
        if (e != cudaSuccess) break;
        if ((e = alloc(h, &C.b, C.cout)) == cudaSuccess && (e = alloc(h, &C.gb, C.cout)) == cudaSuccess &&
            (e = alloc(h, &C.mb, C.cout)) == cudaSuccess && (e = alloc(h, &C.vb, C.cout)) == cudaSuccess) {
            cudaMemset(C.b, 0, sizeof(float) * C.cout);
            cudaMemset(C.mb, 0, sizeof(float) * C.cout);
            e = cudaMemset(C.vb, 0, sizeof(float) * C.cout);
        }
    }
    if (e == cudaSuccess) {
        std::vector<float> wh(17);
        for (int c = 0; c < 16; ++c) wh[c] = nd(rng) * 0.25f;
        wh[16] = 0.f;
        if ((e = alloc(h, &h->wh, 17)) == cudaSuccess && (e = alloc(h, &h->gwh, 17)) == cudaSuccess &&
            (e = alloc(h, &h->mwh, 17)) == cudaSuccess && (e = alloc(h, &h->vwh, 17)) == cudaSuccess) {
            cudaMemcpy(h->wh, wh.data(), sizeof(float) * 17, cudaMemcpyHostToDevice);
            cudaMemset(h->mwh, 0, sizeof(float) * 17);
            e = cudaMemset(h->vwh, 0, sizeof(float) * 17);
        }
    }
    const long n0 = (long)nx * ny * nz, n1 = n0 / 8, n2 = n0 / 64;
    struct Buf { bf16** p; long n; };
    const Buf bufs[] = {{&h->in16, n0 * 16}, {&h->a1, n0 * 16},  {&h->s1, n0 * 16},   {&h->p1, n1 * 16},
                        {&h->a2, n1 * 32},   {&h->s2, n1 * 32},  {&h->p2, n2 * 32},   {&h->a3, n2 * 64},
                        {&h->e3, n2 * 64},   {&h->u2, n1 * 64},  {&h->a4, n1 * 32},   {&h->e2, n1 * 32},
                        {&h->u1, n0 * 32},   {&h->a5, n0 * 16},  {&h->e1, n0 * 16},   {&h->g_e1, n0 * 16},
                        {&h->g_a5, n0 * 16}, {&h->g_s1p, n0 * 16}, {&h->g_u1, n0 * 32}, {&h->g_e2, n1 * 32},
                        {&h->g_a4, n1 * 32}, {&h->g_s2p, n1 * 32}, {&h->g_u2, n1 * 64}, {&h->g_e3, n2 * 64},
                        {&h->g_a3, n2 * 64}, {&h->g_p2, n2 * 32}, {&h->g_s2, n1 * 32},  {&h->g_a2, n1 * 32},
                        {&h->g_p1, n1 * 16}, {&h->g_s1, n0 * 16}, {&h->g_a1, n0 * 16}};
    for (const Buf& b : bufs)
        if (e == cudaSuccess) e = alloc(h, b.p, b.n);
    if (e == cudaSuccess) e = alloc(h, &h->pred, n0);
    if (e == cudaSuccess) e = alloc(h, &h->gpred, n0);
    if (e == cudaSuccess) e = alloc(h, &h->acc, 4);
    if (e != cudaSuccess) {
        wp_set_cuda_error(e, "unet create", __FILE__, __LINE__);
        wp_unet_destroy(h);
        return WP_ERR_CUDA;
    }
    wp_status st = refresh_copies(h, nullptr);
    if (st == WP_OK && (e = cudaDeviceSynchronize()) != cudaSuccess) {
        wp_set_cuda_error(e, "unet create", __FILE__, __LINE__);
        st = WP_ERR_CUDA;
    }
    if (st != WP_OK) { wp_unet_destroy(h); return st; }
    *out = h;
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_unet_predict(wp_unet* h, float* p, const float* b, const float* sdf, double hcell,
                                                void* stream) {
    if (!h || !p || !b || !sdf || !(hcell > 0)) { wp_set_error_msg("wp_unet_predict: bad arguments"); return WP_ERR_INVALID_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    wp_status st = forward(h, b, sdf, hcell, p, s);
    if (st != WP_OK) return st;
    return wp_conv_check_error(s);
}

extern "C" CUWHHD_API wp_status wp_unet_train_step(wp_unet* h, const float* b, const float* sdf, const float* p,
                                                   double hcell, double lr, double* loss, void* stream) {
    if (!h || !b || !sdf || !p || !(hcell > 0) || !(lr >= 0)) {
        wp_set_error_msg("wp_unet_train_step: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    wp_status st = forward(h, b, sdf, hcell, nullptr, s);
    if (st == WP_OK) st = backward(h, sdf, p, hcell, s);
    if (st == WP_OK && lr > 0) st = adam(h, lr, s);
    if (st != WP_OK) return st;
    if ((st = wp_conv_check_error(s)) != WP_OK) return st;
    if (loss) {
        double a[4];
        WP_CUDA_TRY(cudaMemcpyAsync(a, h->acc, sizeof(a), cudaMemcpyDeviceToHost, s));
        WP_CUDA_TRY(cudaStreamSynchronize(s));
        *loss = a[3];
    }
    return WP_OK;
}

// Parameters (which = 0) or gradients of the last step (which = 1) as one FP32 host vector in a
// fixed order: per convolution its part weights [27][cout][cin_p] then its bias, then the head
// (16 weights, bias).  With host == NULL only *count is written.
extern "C" CUWHHD_API wp_status wp_unet_params(wp_unet* h, int which, float* host, size_t cap, size_t* count) {
    if (!h || !count) { wp_set_error_msg("wp_unet_params: null pointer"); return WP_ERR_INVALID_ARG; }
    size_t total = 0;
    each_param(h, [&](float*, float*, long n) { total += (size_t)n; });
    *count = total;
    if (!host) return WP_OK;
    if (cap < total) { wp_set_error_msg("wp_unet_params: buffer too small"); return WP_ERR_INVALID_ARG; }
    size_t off = 0;
    cudaError_t e = cudaDeviceSynchronize();
    each_param(h, [&](float* w, float* g, long n) {
        if (e == cudaSuccess) e = cudaMemcpy(host + off, which ? g : w, sizeof(float) * n, cudaMemcpyDeviceToHost);
        off += (size_t)n;
    });
    if (e != cudaSuccess) { wp_set_cuda_error(e, "wp_unet_params", __FILE__, __LINE__); return WP_ERR_CUDA; }
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_unet_set_params(wp_unet* h, const float* host, size_t count) {
    if (!h || !host) { wp_set_error_msg("wp_unet_set_params: null pointer"); return WP_ERR_INVALID_ARG; }
    size_t total = 0;
    each_param(h, [&](float*, float*, long n) { total += (size_t)n; });
    if (count != total) { wp_set_error_msg("wp_unet_set_params: wrong parameter count"); return WP_ERR_INVALID_ARG; }
    size_t off = 0;
    cudaError_t e = cudaDeviceSynchronize();
    each_param(h, [&](float* w, float*, long n) {
        if (e == cudaSuccess) e = cudaMemcpy(w, host + off, sizeof(float) * n, cudaMemcpyHostToDevice);
        off += (size_t)n;
    });
    if (e != cudaSuccess) { wp_set_cuda_error(e, "wp_unet_set_params", __FILE__, __LINE__); return WP_ERR_CUDA; }
    wp_status st = refresh_copies(h, nullptr);
    if (st == WP_OK && (e = cudaDeviceSynchronize()) != cudaSuccess) {
        wp_set_cuda_error(e, "wp_unet_set_params", __FILE__, __LINE__);
        return WP_ERR_CUDA;
    }
    return st;
}

extern "C" CUWHHD_API wp_status wp_unet_destroy(wp_unet* h) {
    if (!h) return WP_OK;
    cudaDeviceSynchronize();
    for (void* p : h->allocs) cudaFree(p);
    delete h;
    return WP_OK;
}
