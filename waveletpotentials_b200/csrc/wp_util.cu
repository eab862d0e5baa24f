// wp_util.cu -- error reporting and device queries shared by the C ABI.
#include "wp_common.cuh"

#include <cstdint>

#include <cstdio>
#include <cstring>

namespace {
thread_local char g_err[512] = "";
int g_sms[64] = {0};
}  // namespace

void wp_set_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
    snprintf(g_err, sizeof(g_err), "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}

void wp_set_error_msg(const char* msg) { snprintf(g_err, sizeof(g_err), "%s", msg); }

int wp_sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (dev < 64 && g_sms[dev] > 0) return g_sms[dev];
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
    if (dev < 64) g_sms[dev] = sms;
    return sms;
}

extern "C" CUWHHD_API const char* wp_last_error(void) { return g_err; }

extern "C" CUWHHD_API int wp_version(void) { return 1; }

// ---------------------------------------------------------------------------------------------
// Test-only withheld arrival: the next launch at the armed site leaves one wait without the arrival
// it waits for, so that wait runs out after the given limit.  One shot: taking it disarms it; a launch
// that is being captured into a graph does not take it.
#include <mutex>

namespace {
std::mutex g_wh_mu;
int g_wh_site = 0, g_wh_at = 0;
unsigned long long g_wh_ns = 0;
}  // namespace

bool wp_take_withhold(int site, cudaStream_t s, int* at, unsigned long long* limit_ns) {
    // never into a captured graph: every replay would withhold again
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return false;
    std::lock_guard<std::mutex> lk(g_wh_mu);
    if (g_wh_site == 0 || g_wh_site != site) return false;
    *at = g_wh_at;
    *limit_ns = g_wh_ns;
    g_wh_site = 0;
    return true;
}

extern "C" CUWHHD_API wp_status wp_debug_withhold_wait(int site, int at, double limit_seconds) {
    if (site < 0 || site > WP_WAIT_SITE_BATCH_PUBLISH || at < 0 || !(limit_seconds >= 1e-6 && limit_seconds <= 2.0)) {
        wp_set_error_msg("wp_debug_withhold_wait: site 0..3, at >= 0, limit in [1e-6, 2] s");
        return WP_ERR_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lk(g_wh_mu);
    g_wh_site = site;
    g_wh_at = at;
    g_wh_ns = (unsigned long long)(limit_seconds * 1e9);
    return WP_OK;
}

// ---------------------------------------------------------------------------------------------
// Launch accounting and optional per-kernel-class timing with CUDA events recorded on the
// launching stream.  Counting is always on (one relaxed atomic per launch); event timing only
// between wp_profile_enable(1) and wp_profile_enable(0).
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

namespace {
struct ProfRec {
    const char* name;
    cudaEvent_t a, b;
    double bytes;
};
std::atomic<long long> g_launches{0};
std::atomic<bool> g_prof_on{false};
std::mutex g_prof_mu;
std::vector<ProfRec> g_open;   // indexed by token
std::vector<ProfRec> g_done;
std::vector<cudaEvent_t> g_pool;

cudaEvent_t take_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

struct Agg {
    std::string name;
    long long launches = 0;
    double ms = 0.0;
    double bytes = 0.0;
};
std::vector<Agg> g_agg;
}  // namespace

void wp_add_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {
__global__ void read_small_kernel(unsigned int* __restrict__ dst, const unsigned int* __restrict__ src, size_t words) {
    for (size_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
}
struct SmallBuf {
    void* host = nullptr; // mapped page-locked staging
    void* dev = nullptr;  // its device address
    size_t cap = 0;
    ~SmallBuf() {
        if (host) cudaFreeHost(host);
    }
};
}  // namespace

cudaError_t wp_read_small(void* host, const void* dev, size_t bytes, cudaStream_t s) {
    // one staging buffer per host thread (each call completes before returning), mapped and portable
    // so that a kernel on any device stores into it: the readback then takes no copy engine, and a
    // large transfer that another stream has queued on the engines cannot delay it
    thread_local SmallBuf buf;
    if (bytes == 0) return cudaSuccess;
    if (buf.cap < bytes) {
        if (buf.host) cudaFreeHost(buf.host);
        buf.host = buf.dev = nullptr;
        buf.cap = 0;
        const size_t cap = bytes < 4096 ? 4096 : (bytes + 3) / 4 * 4;
        if (cudaHostAlloc(&buf.host, cap, cudaHostAllocMapped | cudaHostAllocPortable) == cudaSuccess &&
            cudaHostGetDevicePointer(&buf.dev, buf.host, 0) == cudaSuccess) {
            buf.cap = cap;
        } else {
            if (buf.host) cudaFreeHost(buf.host);
            buf.host = buf.dev = nullptr;
        }
        (void)cudaGetLastError();
    }
    cudaError_t e;
    if (buf.cap >= bytes && bytes % 4 == 0 && ((uintptr_t)dev & 3u) == 0) {
        read_small_kernel<<<1, 128, 0, s>>>((unsigned int*)buf.dev, (const unsigned int*)dev, bytes / 4);
        wp_add_launches(1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess) memcpy(host, buf.host, bytes);
    } else {
        e = cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    return e;
}

int wp_prof_start(cudaStream_t s) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (!g_prof_on.load(std::memory_order_relaxed)) return -1;
    // launches captured into a graph are not timed one by one (their events would only fire at
    // replay); the graph launch is timed as a whole by its owner
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return -1;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    ProfRec r{nullptr, take_event(), take_event(), 0.0};
    cudaEventRecord(r.a, s);
    g_open.push_back(r);
    return (int)g_open.size() - 1;
}

void wp_prof_stop(int tok, const char* name, double bytes, cudaStream_t s) {
    if (tok < 0) return;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (tok >= (int)g_open.size()) return;
    ProfRec& r = g_open[tok];
    r.name = name;
    r.bytes = bytes;
    cudaEventRecord(r.b, s);
}

extern "C" CUWHHD_API void wp_profile_enable(int on) { g_prof_on.store(on != 0); }

bool wp_profile_is_enabled() { return g_prof_on.load(); }

extern "C" CUWHHD_API void wp_profile_reset(void) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (auto& r : g_open) { g_pool.push_back(r.a); g_pool.push_back(r.b); }
    g_open.clear();
    g_agg.clear();
    g_launches.store(0);
}

extern "C" CUWHHD_API long long wp_launch_count(void) { return g_launches.load(); }

// Synchronizes the device, folds the recorded events into per-name totals and returns the
// number of kernel classes; wp_profile_entry(i, ...) reads them.
extern "C" CUWHHD_API int wp_profile_collect(void) {
    cudaDeviceSynchronize();
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (auto& r : g_open) {
        float ms = 0.f;
        if (r.name && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
            Agg* a = nullptr;
            for (auto& x : g_agg) if (x.name == r.name) { a = &x; break; }
            if (!a) { g_agg.push_back(Agg{r.name}); a = &g_agg.back(); }
            a->launches += 1;
            a->ms += ms;
            a->bytes += r.bytes;
        }
        g_pool.push_back(r.a);
        g_pool.push_back(r.b);
    }
    g_open.clear();
    return (int)g_agg.size();
}

extern "C" CUWHHD_API int wp_profile_entry(int i, char* name, int name_cap, long long* launches, double* ms,
                                           double* bytes) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (i < 0 || i >= (int)g_agg.size()) return 1;
    const Agg& a = g_agg[i];
    if (name && name_cap > 0) snprintf(name, name_cap, "%s", a.name.c_str());
    if (launches) *launches = a.launches;
    if (ms) *ms = a.ms;
    if (bytes) *bytes = a.bytes;
    return 0;
}

#include <map>
#include <utility>

cudaError_t wp_set_smem_impl(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair(kernel, dev);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) done[key] = bytes;
    return e;
}

// ---------------------------------------------------------------------------------------------
// TMA tensor maps (the driver entry point is resolved once per process)
#include "wp_tc.cuh"

namespace wptc {
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

bool map_f32_3d(CUtensorMap* m, const float* base, int n0, int n1, int n2, int b0, int b1) {
    EncodeTiledFn fn = encode_tiled();
    if (!fn || ((uintptr_t)base & 15u) || (n0 * 4) % 16 || (b0 * 4) % 16) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)n0, (cuuint64_t)n1, (cuuint64_t)n2};
    const cuuint64_t strides[2] = {(cuuint64_t)n0 * 4, (cuuint64_t)n0 * 4 * n1};
    const cuuint32_t box[3] = {(cuuint32_t)b0, (cuuint32_t)b1, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace wptc
