// wp_common.cuh -- shared definitions for the sm_100a WaveletPotentials kernels.
//
// Layout (the reference's, Utils.h:46-47): element (x, y, z) of an array with extents
// (DX, DY, DZ) lives at y + x*DY + z*DX*DY; y is contiguous.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/wp_api.h"

#define WP_CUDA_TRY(expr)                                   \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) { wp_set_cuda_error(_e, #expr, __FILE__, __LINE__); return WP_ERR_CUDA; } \
    } while (0)

#define WP_LAUNCH_CHECK()                                   \
    do {                                                    \
        cudaError_t _e = cudaGetLastError();                \
        if (_e != cudaSuccess) { wp_set_cuda_error(_e, "kernel launch", __FILE__, __LINE__); return WP_ERR_CUDA; } \
    } while (0)

void wp_set_cuda_error(cudaError_t e, const char* what, const char* file, int line);
void wp_set_error_msg(const char* msg);

// wavelet ids (same values as the reference enum, WaveletTypes.h:7-27)
enum { WP_ID_CDF3_5 = 2, WP_ID_CDF2_6 = 5, WP_ID_CDF4_4 = 6, WP_ID_CDF4_6 = 7, WP_ID_CDF2_8 = 10, WP_ID_CDF3_7 = 11,
       WP_ID_CDF2_0 = 16, WP_ID_CDF1_1 = 17, WP_ID_CDF1_7 = 18 };

static inline int wp_ilog2(int n) {
    int l = 0;
    while ((1 << (l + 1)) <= n) ++l;
    return l;
}
static inline bool wp_is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
static inline int wp_half_up(int n) { return (n & 1) ? (n >> 1) + 1 : (n >> 1); }
static inline unsigned wp_cdiv(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// Test-only withheld arrival armed by wp_debug_withhold_wait for `site`: true once (then disarmed),
// with the index of the withheld arrival and the wait limit in nanoseconds; never while s is capturing.
bool wp_take_withhold(int site, cudaStream_t s, int* at, unsigned long long* limit_ns);

// Number of SMs of the current device (cached per process; 148 on B200).
int wp_sm_count();

// Launch accounting (always) and per-kernel-class event timing (when enabled): wrap a launch as
//   WP_KERNEL("name", algorithmic_bytes, stream, kernel<<<g, b, smem, stream>>>(...));
int wp_prof_start(cudaStream_t s);
// Launch-count adjustment for work replayed from a CUDA graph (captured launches are counted once at
// capture time; a replay adds them again).
void wp_add_launches(long long n);
// Reads a few bytes of device memory into host memory, ordered on stream s (synchronous).  A kernel
// stores them into a mapped page-locked buffer, so the readback takes no copy engine and never
// queues behind a large transfer another stream has in flight.
cudaError_t wp_read_small(void* host, const void* dev, size_t bytes, cudaStream_t s);
bool wp_profile_is_enabled();
template <typename T>
wp_status wp_dwt_axis_tune(T* buf, int DX, int DY, int DZ, int levels, char axis, int wavelet, char bc, int forward,
                           cudaStream_t s);
// Uploads the wavelet filter tables to the current device (once; synchronous).
cudaError_t wp_dwt_prepare();
void wp_prof_stop(int tok, const char* name, double bytes, cudaStream_t s);
#define WP_KERNEL(name, bytes, stream, ...)                         \
    do {                                                            \
        const int _tok = wp_prof_start(stream);                     \
        __VA_ARGS__;                                                \
        WP_LAUNCH_CHECK();                                          \
        wp_prof_stop(_tok, name, (double)(bytes), stream);          \
    } while (0)

// Programmatic dependent launch.  A kernel that calls wp_pdl_enter() first waits until the grid
// launched before it on the stream has completed and its memory is visible (griddepcontrol.wait;
// immediate when there is no programmatic dependency), then lets the grid after it be scheduled
// (griddepcontrol.launch_dependents) -- that grid's CTAs become resident as this grid's last wave
// drains, hiding launch latency and tails.  wp_launch_pdl launches with the attribute that allows
// it (kernel-to-kernel only; on the legacy default stream it launches normally).
__device__ __forceinline__ void wp_pdl_enter() {
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 900)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" :::);
#endif
}

template <typename... KArgs, typename... Args>
void wp_launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    if (s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread) {
        kern<<<grid, block, smem, s>>>(static_cast<KArgs>(args)...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    (void)cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// Raises a kernel's dynamic shared-memory limit once per (kernel, device) (a host-side attribute
// call, kept out of the launch path so launches can be captured into CUDA graphs).
cudaError_t wp_set_smem_impl(const void* kernel, size_t bytes);
template <typename K>
cudaError_t wp_set_smem(K kernel, size_t bytes) {
    return wp_set_smem_impl(reinterpret_cast<const void*>(kernel), bytes);
}

// transform along one axis (wp_dwt.cu); T = float or double
template <typename T>
wp_status wp_dwt_axis_launch(T* dst, const T* src, int DX, int DY, int DZ, int levels, char axis, int wavelet,
                             char bc, int forward, cudaStream_t stream);
