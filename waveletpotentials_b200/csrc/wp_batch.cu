// wp_batch.cu -- many independent projections of uneven sizes (2D and 3D) in one CUDA-graph launch.
//
// No reference counterpart (the reference runs one grid per process).  The whole batch --
// divergence, tolerance-driven mixed-precision solve, gradient update, max|div|, wavelet recovery
// for every grid -- is captured once into a CUDA graph with the grids spread over `nstreams`
// concurrent branches, and replayed with one cudaGraphLaunch.  Each grid's solve is a device-side
// loop (a while-node whose body is one refinement step and whose test kernel applies the stopping
// rule), so every replay runs as many steps as that grid's current input needs.  An optional eager
// plan pass (wp_batch_plan) measures the step counts of a representative input; they only order the
// grids over the branches (costliest first).  Per-grid max|div|, the final FP64 relative residual and
// the V-cycle count stay on the device until wp_batch_results() reads them with one copy.
// In WP_BATCH_PERSISTENT mode the solves of all grids run instead in one persistent kernel inside the
// graph (wp_mg.cu, batch_persist_kernel: a device work queue of (grid, level, pass) tiles), between
// the grids' divergences and their gradient updates and recoveries on the branches.
#include "wp_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <new>
#include <vector>

struct wp_mgfrac2d;
wp_status wp_mg_prepare_mixed(wp_mgfrac3d* h);
wp_status wp_mg_solve_mixed_loop_capture(wp_mgfrac3d* h, float* dst, const float* f, const wp_mg_params* prm,
                                         cudaStream_t s, long long* body_launches);
const void* wp_mg_loop_state(const wp_mgfrac3d* h);
void wp_mg_forbid_persistent(wp_mgfrac3d* h);
wp_status wp_mg_solve_tol_internal(wp_mgfrac3d* h, float* dst, const float* f, const wp_mg_params* prm, wp_mg_report* r,
                                   cudaStream_t s);
const double* wp_mg_slots(const wp_mgfrac3d* h);
const double* wp_mg_p64(const wp_mgfrac3d* h);
wp_mgfrac3d* wp_mg2d_impl(wp_mgfrac2d* h);
wp_status wp_max_abs_device(const float* x, size_t n, unsigned int* d_out, cudaStream_t s);
struct wp_mg_pbatch;
wp_status wp_mg_pbatch_create(wp_mg_pbatch** out, wp_mgfrac3d* const* hs, float* const* dst, const float* const* f,
                              int count, const wp_mg_params* prm, long target_cells);
wp_status wp_mg_pbatch_arm(wp_mg_pbatch* pb, int at, unsigned long long limit_ns, cudaStream_t s);
wp_status wp_mg_pbatch_launch(wp_mg_pbatch* pb, cudaStream_t s);
void wp_mg_pbatch_destroy(wp_mg_pbatch* pb);
wp_status wp_mg_pbatch_profile(wp_mg_pbatch* pb, int enable, unsigned long long* out, cudaStream_t s);
int wp_mg_pbatch_prof_slots();

namespace {

struct Grid {
    int dims;
    int n[3];
    double h;
    const float* frac[3];
    wp_mgfrac3d* mg3 = nullptr;
    wp_mgfrac2d* mg2 = nullptr;
    wp_recover3d* rec3 = nullptr;
    wp_recover2d* rec2 = nullptr;
    float* b = nullptr;
    float* p = nullptr;
    int cycles = 0;               // V-cycles of the plan's eager solve (orders the branches)
    long long body_launches = 0;  // kernels in one pass of the captured loop body
    long cells() const { return (long)n[0] * n[1] * n[2]; }
    wp_mgfrac3d* mg() const { return dims == 3 ? mg3 : wp_mg2d_impl(mg2); }
};

constexpr int kOut = 5;  // per-grid results
// per grid: max|div|, the FP64 relative residual of the last refinement step, the MG handle's device
// error flag (the int after its four norm slots; nonzero when a bounded wait gave up), and the
// device loop's V-cycle and refinement-step counts (ints 0 and 4 of its state)
__global__ void gather_results_kernel(double* out, const double* const* slots, const int* const* loops,
                                      const unsigned* maxbits, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const double* a = slots[i];
    out[kOut * i] = (double)__uint_as_float(maxbits[i]);
    out[kOut * i + 1] = a[1] > 0.0 ? sqrt(a[0] / a[1]) : 0.0;
    out[kOut * i + 2] = (double)*reinterpret_cast<const int*>(a + 4);
    out[kOut * i + 3] = (double)loops[i][0];
    out[kOut * i + 4] = (double)loops[i][4];
}

}  // namespace

struct wp_batch {
    std::vector<Grid> g;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    wp_mg_params prm;
    unsigned* d_max = nullptr;       // per grid: max|div| bits
    const double** d_slots = nullptr; // per grid: pointer to the MG handle's norm slots
    const int** d_loops = nullptr;   // per grid: pointer to the MG handle's device loop state
    double* d_out = nullptr;         // per grid: kOut results (see gather_results_kernel)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<const void*> bound;  // pointers captured into the graph
    long long graph_launches = 0;    // kernels in one replay of the graph outside the loop bodies
    bool planned = false;
    bool counted = true;             // the last replay's loop-body kernels were added to the count
    int mode = WP_BATCH_GRAPH;       // as asked: WP_BATCH_GRAPH, WP_BATCH_PERSISTENT or WP_BATCH_AUTO
    int run_mode = WP_BATCH_GRAPH;   // as run (AUTO: the plan's choice, the graph mode before a plan)
    float graph_ms = 0.f;            // AUTO: the plan's timing of the graph mode's solves (0 = not timed)
    long long tile_cells = 0;        // persistent mode: cells per work-queue tile (0 = default)
    bool tile_auto = true;           // the caller left the tile to the library: wp_batch_plan tunes it
    float tile_ms[5] = {0.f, 0.f, 0.f, 0.f, 0.f};  // the tuner's timings of kTileCands (0 = not timed)
    wp_mg_pbatch* pb = nullptr;      // persistent mode: every grid's solve program, in cost order
    bool pers_ok = true;             // AUTO: the grids fit the persistent program
};

namespace {

// b = -div(a u) of grid i (the solve's right-hand side)
wp_status divergence_one(wp_batch* B, int i, const float* xv, const float* yv, const float* zv, cudaStream_t s) {
    Grid& G = B->g[i];
    const double h = G.h;
    if (G.dims == 3)
        return wp_divergence_frac3d(G.b, xv, yv, zv, G.frac[0], G.frac[1], G.frac[2], G.n[0], G.n[1], G.n[2], h, h, h,
                                    s);
    return wp_divergence_frac2d(G.b, xv, yv, G.frac[0], G.frac[1], G.n[0], G.n[1], h, h, s);
}

// after the solve: u <- (u - grad p) a, max|div u|, wavelet potential recovery
wp_status finish_one(wp_batch* B, int i, float* xv, float* yv, float* zv, float* qx, float* qy, float* qz,
                     cudaStream_t s) {
    Grid& G = B->g[i];
    wp_status st;
    const double h = G.h;
    if (G.dims == 3) {
        // the gradient of the FP64 iterate, formed in FP64 (as the one-grid projector does)
        if ((st = wp_grad_subtract_frac3d_p64(xv, yv, zv, wp_mg_p64(G.mg3), G.frac[0], G.frac[1], G.frac[2], G.n[0],
                                              G.n[1], G.n[2], h, h, h, 1, s)) != WP_OK)
            return st;
        if ((st = wp_divergence_frac3d(G.b, xv, yv, zv, nullptr, nullptr, nullptr, G.n[0], G.n[1], G.n[2], h, h, h, s)) !=
            WP_OK)
            return st;
        if ((st = wp_max_abs_device(G.b, G.cells(), B->d_max + i, s)) != WP_OK) return st;
        return wp_recover3d_run(G.rec3, qx, qy, qz, xv, yv, zv, s);
    }
    if ((st = wp_grad_subtract_frac2d(xv, yv, G.p, G.frac[0], G.frac[1], G.n[0], G.n[1], h, h, 1, s)) != WP_OK) return st;
    if ((st = wp_divergence_frac2d(G.b, xv, yv, nullptr, nullptr, G.n[0], G.n[1], h, h, s)) != WP_OK) return st;
    if ((st = wp_max_abs_device(G.b, G.cells(), B->d_max + i, s)) != WP_OK) return st;
    return wp_recover2d_run(G.rec2, qz, xv, yv, s);
}

// one grid on one branch: divergence, its device-loop solve, the rest
wp_status project_one(wp_batch* B, int i, float* xv, float* yv, float* zv, float* qx, float* qy, float* qz,
                      cudaStream_t s) {
    Grid& G = B->g[i];
    wp_status st;
    if ((st = divergence_one(B, i, xv, yv, zv, s)) != WP_OK) return st;
    if ((st = wp_mg_solve_mixed_loop_capture(G.mg(), G.p, G.b, &B->prm, s, &G.body_launches)) != WP_OK) return st;
    return finish_one(B, i, xv, yv, zv, qx, qy, qz, s);
}

// costliest grids first: cells x (planned V-cycles + 2), or cells alone without a plan
std::vector<int> cost_order(const wp_batch* B) {
    const int count = (int)B->g.size();
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    auto cost = [&](int i) { return B->g[i].cells() * (B->planned ? B->g[i].cycles + 2 : 1); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    return order;
}

// the persistent solve of every grid, programs in cost order
wp_status build_pbatch(wp_batch* B) {
    if (B->pb) return WP_OK;
    const std::vector<int> order = cost_order(B);
    std::vector<wp_mgfrac3d*> hs;
    std::vector<float*> dst;
    std::vector<const float*> f;
    for (int i : order) {
        hs.push_back(B->g[i].mg());
        dst.push_back(B->g[i].p);
        f.push_back(B->g[i].b);
    }
    return wp_mg_pbatch_create(&B->pb, hs.data(), dst.data(), f.data(), (int)order.size(), &B->prm,
                               (long)B->tile_cells);
}

void destroy_graph(wp_batch* B) {
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    B->exec = nullptr;
    B->graph = nullptr;
    B->bound.clear();
}

}  // namespace

extern "C" CUWHHD_API wp_status wp_batch_create(wp_batch** out, int count, const int* dims, const int* ext,
                                                const double* dx, const float* const* ax, const float* const* ay,
                                                const float* const* az, const wp_mg_params* prm, int nstreams) {
    if (!out) { wp_set_error_msg("wp_batch_create: null handle"); return WP_ERR_INVALID_ARG; }
    *out = nullptr;
    if (count <= 0 || !dims || !ext || !dx || !ax || !ay || !prm || nstreams < 1 || nstreams > 64) {
        wp_set_error_msg("wp_batch_create: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    wp_batch* B = new (std::nothrow) wp_batch();
    if (!B) return WP_ERR_INVALID_ARG;
    B->prm = *prm;
    B->g.resize(count);
    wp_status st = WP_OK;
    for (int i = 0; i < count && st == WP_OK; ++i) {
        Grid& G = B->g[i];
        G.dims = dims[i];
        G.n[0] = ext[3 * i];
        G.n[1] = ext[3 * i + 1];
        G.n[2] = dims[i] == 3 ? ext[3 * i + 2] : 1;
        G.h = dx[i];
        G.frac[0] = ax[i];
        G.frac[1] = ay[i];
        G.frac[2] = dims[i] == 3 && az ? az[i] : nullptr;
        if (G.dims == 3) {
            if ((st = wp_mgfrac3d_create(&G.mg3, ax[i], ay[i], G.frac[2], G.n[0], G.n[1], G.n[2], G.h, G.h, G.h, 'n',
                                         nullptr)) != WP_OK)
                break;
            wp_mg_forbid_persistent(G.mg3);
            if ((st = wp_recover3d_create(&G.rec3, G.n[0], G.n[1], G.n[2], G.h, G.h, G.h, 'n', WP_CDF3_7, WP_CDF4_6)) !=
                WP_OK)
                break;
        } else if (G.dims == 2) {
            if ((st = wp_mgfrac2d_create(&G.mg2, ax[i], ay[i], G.n[0], G.n[1], G.h, G.h, 'n', nullptr)) != WP_OK) break;
            wp_mg_forbid_persistent(wp_mg2d_impl(G.mg2));
            if ((st = wp_recover2d_create(&G.rec2, G.n[0], G.n[1], G.h, G.h, 'n', WP_CDF3_7, WP_CDF4_6)) != WP_OK) break;
        } else {
            wp_set_error_msg("wp_batch_create: dims must be 2 or 3");
            st = WP_ERR_INVALID_ARG;
            break;
        }
        if ((st = wp_mg_prepare_mixed(G.mg())) != WP_OK) break;
        if ((st = wp_mgfrac3d_autotune(G.mg(), nullptr)) != WP_OK) break;
        cudaError_t e = cudaMalloc((void**)&G.b, sizeof(float) * G.cells());
        if (e == cudaSuccess) e = cudaMalloc((void**)&G.p, sizeof(float) * G.cells());
        if (e != cudaSuccess) { wp_set_cuda_error(e, "batch alloc", __FILE__, __LINE__); st = WP_ERR_CUDA; }
    }
    if (st == WP_OK) {
        B->streams.resize(nstreams);
        B->events.resize(nstreams + 1);
        for (auto& s : B->streams) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        for (auto& e : B->events) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        std::vector<const double*> slots(count);
        std::vector<const int*> loops(count);
        for (int i = 0; i < count; ++i) {
            slots[i] = wp_mg_slots(B->g[i].mg());
            loops[i] = reinterpret_cast<const int*>(wp_mg_loop_state(B->g[i].mg()));
        }
        cudaError_t e = cudaMalloc((void**)&B->d_max, sizeof(unsigned) * count);
        if (e == cudaSuccess) e = cudaMalloc((void**)&B->d_slots, sizeof(double*) * count);
        if (e == cudaSuccess) e = cudaMalloc((void**)&B->d_loops, sizeof(int*) * count);
        if (e == cudaSuccess) e = cudaMalloc((void**)&B->d_out, sizeof(double) * kOut * count);
        if (e == cudaSuccess) e = cudaMemcpy(B->d_slots, slots.data(), sizeof(double*) * count, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(B->d_loops, loops.data(), sizeof(int*) * count, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { wp_set_cuda_error(e, "batch alloc", __FILE__, __LINE__); st = WP_ERR_CUDA; }
    }
    if (st != WP_OK) { wp_batch_destroy(B); return st; }
    *out = B;
    return WP_OK;
}

namespace {

constexpr int kTileN = 5;
constexpr long long kTileCands[kTileN] = {4096, 8192, 16384, 32768, 65536};

// Persistent mode, tile left to the library: the persistent solve of the plan's right-hand sides
// timed with each candidate tile (one warm-up launch, one timed), the fastest kept.
wp_status tune_tiles(wp_batch* B, cudaStream_t s) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    WP_CUDA_TRY(cudaEventCreate(&e0));
    WP_CUDA_TRY(cudaEventCreate(&e1));
    wp_status st = WP_OK;
    float best = 0.f;
    long long pick = 0;
    for (int k = 0; k < kTileN && st == WP_OK; ++k) {
        if (B->pb) wp_mg_pbatch_destroy(B->pb);
        B->pb = nullptr;
        B->tile_cells = kTileCands[k];
        if ((st = build_pbatch(B)) != WP_OK) break;
        if ((st = wp_mg_pbatch_launch(B->pb, s)) != WP_OK) break;
        cudaEventRecord(e0, s);
        if ((st = wp_mg_pbatch_launch(B->pb, s)) != WP_OK) break;
        cudaEventRecord(e1, s);
        cudaError_t e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) {
            wp_set_cuda_error(e, "batch tile tuning", __FILE__, __LINE__);
            st = WP_ERR_CUDA;
            break;
        }
        B->tile_ms[k] = ms;
        if (pick == 0 || ms < best) {
            best = ms;
            pick = kTileCands[k];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (B->pb) wp_mg_pbatch_destroy(B->pb);
    B->pb = nullptr;  // rebuilt with the chosen tile at the next capture
    if (pick) B->tile_cells = pick;
    return st;
}

// AUTO: the solves of every grid as the graph mode runs them (a device loop per grid, round-robin
// over the branches, on the plan's right-hand sides), captured once, replayed once to warm up and
// once timed.
wp_status time_graph_solves(wp_batch* B, cudaStream_t s, float* ms_out) {
    const std::vector<int> order = cost_order(B);
    const size_t ns = B->streams.size();
    cudaStream_t cs = B->streams[0];
    const long long c0 = wp_launch_count();
    WP_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaEventRecord(B->events[0], cs);
    for (size_t k = 1; k < ns; ++k) cudaStreamWaitEvent(B->streams[k], B->events[0], 0);
    wp_status st = WP_OK;
    for (size_t k = 0; k < order.size() && st == WP_OK; ++k) {
        Grid& G = B->g[order[k]];
        long long bl = 0;
        st = wp_mg_solve_mixed_loop_capture(G.mg(), G.p, G.b, &B->prm, B->streams[k % ns], &bl);
    }
    for (size_t k = 1; k < ns; ++k) {
        cudaEventRecord(B->events[k], B->streams[k]);
        cudaStreamWaitEvent(cs, B->events[k], 0);
    }
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(cs, &graph);
    wp_add_launches(-(wp_launch_count() - c0));  // timing only: not the caller's launches
    if (st != WP_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (st != WP_OK) return st;
        wp_set_cuda_error(e, "batch mode timing capture", __FILE__, __LINE__);
        return WP_ERR_CUDA;
    }
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, s);
    if (e == cudaSuccess) e = cudaEventRecord(e0, s);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, s);
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms_out, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (exec) cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        wp_set_cuda_error(e, "batch mode timing", __FILE__, __LINE__);
        return WP_ERR_CUDA;
    }
    return WP_OK;
}

// AUTO: the persistent solve (its tile tuned when the caller left it open) against the graph mode's
// solves, both on the plan's right-hand sides; the faster one runs from now on.
wp_status choose_mode(wp_batch* B, cudaStream_t s) {
    B->run_mode = WP_BATCH_GRAPH;
    if (!B->pers_ok) return WP_OK;
    wp_status st = WP_OK;
    float pers = 0.f;
    if (B->tile_auto) {
        if ((st = tune_tiles(B, s)) != WP_OK) return st;
        for (int k = 0; k < kTileN; ++k)
            if (kTileCands[k] == B->tile_cells) pers = B->tile_ms[k];
    } else {
        if ((st = build_pbatch(B)) != WP_OK) return st;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        WP_CUDA_TRY(cudaEventCreate(&e0));
        WP_CUDA_TRY(cudaEventCreate(&e1));
        if ((st = wp_mg_pbatch_launch(B->pb, s)) == WP_OK) {
            cudaEventRecord(e0, s);
            st = wp_mg_pbatch_launch(B->pb, s);
            cudaEventRecord(e1, s);
        }
        cudaError_t e = cudaEventSynchronize(e1);
        if (e == cudaSuccess && st == WP_OK) e = cudaEventElapsedTime(&pers, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        wp_mg_pbatch_destroy(B->pb);
        B->pb = nullptr;
        if (st != WP_OK) return st;
        if (e != cudaSuccess) {
            wp_set_cuda_error(e, "batch mode timing", __FILE__, __LINE__);
            return WP_ERR_CUDA;
        }
    }
    if ((st = time_graph_solves(B, s, &B->graph_ms)) != WP_OK) return st;
    B->run_mode = pers > 0.f && pers < B->graph_ms ? WP_BATCH_PERSISTENT : WP_BATCH_GRAPH;
    return WP_OK;
}

}  // namespace

// Eager pass: per grid, b = -div(a u) and a tolerance-driven mixed solve; records the V-cycles each
// grid needs on this input (the velocities are not modified), which order the grids over the graph's
// branches.  Optional: without it the grids are ordered by size.  Synchronous.
extern "C" CUWHHD_API wp_status wp_batch_plan(wp_batch* B, const float* const* xv, const float* const* yv,
                                              const float* const* zv, int* cycles_out, void* stream) {
    if (!B || !xv || !yv) { wp_set_error_msg("wp_batch_plan: null pointer"); return WP_ERR_INVALID_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    for (size_t i = 0; i < B->g.size(); ++i) {
        Grid& G = B->g[i];
        wp_status st;
        if (G.dims == 3)
            st = wp_divergence_frac3d(G.b, xv[i], yv[i], zv[i], G.frac[0], G.frac[1], G.frac[2], G.n[0], G.n[1], G.n[2],
                                      G.h, G.h, G.h, s);
        else
            st = wp_divergence_frac2d(G.b, xv[i], yv[i], G.frac[0], G.frac[1], G.n[0], G.n[1], G.h, G.h, s);
        if (st != WP_OK) return st;
        wp_mg_params prm = B->prm;
        prm.precision = WP_PREC_MIXED;
        wp_mg_report rep;
        st = wp_mg_solve_tol_internal(G.mg(), G.p, G.b, &prm, &rep, s);
        if (st != WP_OK && st != WP_ERR_NOT_CONVERGED) return st;
        G.cycles = rep.cycles;
        if (cycles_out) cycles_out[i] = rep.cycles;
    }
    B->planned = true;
    destroy_graph(B);
    // the programs follow the new cost order
    if (B->pb) {
        wp_mg_pbatch_destroy(B->pb);
        B->pb = nullptr;
    }
    if (B->mode == WP_BATCH_PERSISTENT && B->tile_auto) return tune_tiles(B, s);
    if (B->mode == WP_BATCH_AUTO) return choose_mode(B, s);
    return WP_OK;
}

// Runs the whole batch as one CUDA-graph launch (captured on first use or when the pointer set
// changes).  2D grids use xv, yv and qz only.
extern "C" CUWHHD_API wp_status wp_batch_run(wp_batch* B, float* const* xv, float* const* yv, float* const* zv,
                                             float* const* qx, float* const* qy, float* const* qz, void* stream) {
    if (!B || !xv || !yv || !qz) { wp_set_error_msg("wp_batch_run: null pointer"); return WP_ERR_INVALID_ARG; }
    const int count = (int)B->g.size();
    std::vector<const void*> ptrs;
    for (int i = 0; i < count; ++i) {
        const bool d3 = B->g[i].dims == 3;
        if (d3 && (!zv || !qx || !qy || !zv[i] || !qx[i] || !qy[i])) {
            wp_set_error_msg("wp_batch_run: 3D grid without zv/qx/qy");
            return WP_ERR_INVALID_ARG;
        }
        ptrs.insert(ptrs.end(), {xv[i], yv[i], d3 ? zv[i] : nullptr, d3 ? qx[i] : nullptr, d3 ? qy[i] : nullptr, qz[i]});
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (!B->exec || ptrs != B->bound) {
        destroy_graph(B);
        wp_status pst;
        if (B->run_mode == WP_BATCH_PERSISTENT && (pst = build_pbatch(B)) != WP_OK) return pst;
        cudaStream_t cs = B->streams[0];
        const long long launches0 = wp_launch_count();
        WP_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        wp_status st = WP_OK;
        cudaEventRecord(B->events[0], cs);
        for (size_t k = 1; k < B->streams.size(); ++k) cudaStreamWaitEvent(B->streams[k], B->events[0], 0);
        // costliest grids first, round-robin over the branches
        const std::vector<int> order = cost_order(B);
        const size_t ns = B->streams.size();
        auto join = [&]() {
            for (size_t k = 1; k < ns; ++k) {
                cudaEventRecord(B->events[k], B->streams[k]);
                cudaStreamWaitEvent(cs, B->events[k], 0);
            }
        };
        if (B->run_mode == WP_BATCH_PERSISTENT) {
            // divergences on the branches, every solve in the persistent kernel, then the rest
            for (int k = 0; k < count && st == WP_OK; ++k) {
                const int i = order[k];
                st = divergence_one(B, i, xv[i], yv[i], B->g[i].dims == 3 ? zv[i] : nullptr, B->streams[k % ns]);
                B->g[i].body_launches = 0;
            }
            join();
            if (st == WP_OK) st = wp_mg_pbatch_launch(B->pb, cs);
            cudaEventRecord(B->events[0], cs);
            for (size_t k = 1; k < ns; ++k) cudaStreamWaitEvent(B->streams[k], B->events[0], 0);
            for (int k = 0; k < count && st == WP_OK; ++k) {
                const int i = order[k];
                const bool d3 = B->g[i].dims == 3;
                st = finish_one(B, i, xv[i], yv[i], d3 ? zv[i] : nullptr, d3 ? qx[i] : nullptr, d3 ? qy[i] : nullptr,
                                qz[i], B->streams[k % ns]);
            }
        } else {
            for (int k = 0; k < count && st == WP_OK; ++k) {
                const int i = order[k];
                const bool d3 = B->g[i].dims == 3;
                st = project_one(B, i, xv[i], yv[i], d3 ? zv[i] : nullptr, d3 ? qx[i] : nullptr, d3 ? qy[i] : nullptr,
                                 qz[i], B->streams[k % ns]);
            }
        }
        join();
        if (st == WP_OK) {
            const int tok = wp_prof_start(cs);
            gather_results_kernel<<<wp_cdiv(count, 128), 128, 0, cs>>>(B->d_out, B->d_slots, B->d_loops, B->d_max,
                                                                       count);
            wp_prof_stop(tok, "batch_gather", 8.0 * kOut * count, cs);
        }
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(cs, &graph);
        if (e != cudaSuccess || st != WP_OK) wp_add_launches(-(wp_launch_count() - launches0));
        if (st != WP_OK) { if (graph) cudaGraphDestroy(graph); return st; }
        if (e != cudaSuccess) { wp_set_cuda_error(e, "batch capture", __FILE__, __LINE__); return WP_ERR_CUDA; }
        B->graph = graph;
        e = cudaGraphInstantiate(&B->exec, graph, 0);
        if (e != cudaSuccess) { wp_set_cuda_error(e, "batch instantiate", __FILE__, __LINE__); destroy_graph(B); return WP_ERR_CUDA; }
        B->bound = ptrs;
        B->graph_launches = wp_launch_count() - launches0;
        wp_add_launches(-B->graph_launches);
    }
    if (B->run_mode == WP_BATCH_PERSISTENT) {
        // test only: a withheld publication armed for this run (never inside a capture)
        int at = -1;
        unsigned long long lim = 0;
        if (!wp_take_withhold(WP_WAIT_SITE_BATCH_PUBLISH, s, &at, &lim)) {
            at = -1;
            lim = 0;
        }
        wp_status ast;
        if ((ast = wp_mg_pbatch_arm(B->pb, at, lim, s)) != WP_OK) return ast;
    }
    const int tok = wp_prof_start(s);
    wp_add_launches(B->graph_launches - 1);
    B->counted = false;
    const cudaError_t e = cudaGraphLaunch(B->exec, s);
    wp_prof_stop(tok, "batch_graph", 0.0, s);
    if (e != cudaSuccess) { wp_set_cuda_error(e, "batch graph launch", __FILE__, __LINE__); return WP_ERR_CUDA; }
    return WP_OK;
}

// Per grid (max|div| of the projected field, final FP64 relative residual, V-cycles of the last
// replay); synchronous.  Each grid's device loop stops at the tolerance or at max_cycles, so a grid
// whose residual is still above the tolerance (the cycle cap reached, or a non-finite residual) makes
// the call return WP_ERR_NOT_CONVERGED (every output still written).  A bounded device wait that gave
// up in any grid's solve takes precedence (WP_ERR_DEVICE_WAIT; its flag is cleared).
extern "C" CUWHHD_API wp_status wp_batch_results(wp_batch* B, double* max_abs_div, double* rel_residual,
                                                 int* cycles, void* stream) {
    if (!B) { wp_set_error_msg("wp_batch_results: null handle"); return WP_ERR_INVALID_ARG; }
    const int count = (int)B->g.size();
    std::vector<double> out(kOut * count);
    cudaStream_t s = (cudaStream_t)stream;
    WP_CUDA_TRY(wp_read_small(out.data(), B->d_out, sizeof(double) * kOut * count, s));
    WP_CUDA_TRY(cudaStreamSynchronize(s));
    int over = 0, waits = 0;
    for (int i = 0; i < count; ++i) {
        const double* o = out.data() + kOut * i;
        if (max_abs_div) max_abs_div[i] = o[0];
        if (rel_residual) rel_residual[i] = o[1];
        if (cycles) cycles[i] = (int)o[3];
        if (B->prm.rel_tol > 0.0 && !(o[1] <= B->prm.rel_tol)) ++over;
        // the loop bodies of the last replay: their kernels, counted now that the passes are known (a
        // full-multigrid start runs its first step before the loop, in the counted part of the graph)
        if (!B->counted) {
            const long long passes = (long long)o[4] - (B->prm.start == WP_START_FMG ? 1 : 0);
            wp_add_launches(std::max(passes, 0LL) * B->g[i].body_launches);
        }
        if (o[2] != 0.0) {
            ++waits;
            WP_CUDA_TRY(cudaMemsetAsync((void*)(wp_mg_slots(B->g[i].mg()) + 4), 0, sizeof(int), s));
        }
    }
    B->counted = true;
    char msg[160];
    if (waits) {
        WP_CUDA_TRY(cudaStreamSynchronize(s));
        snprintf(msg, sizeof(msg), "wp_batch_results: a bounded device wait gave up in %d grid(s)", waits);
        wp_set_error_msg(msg);
        return WP_ERR_DEVICE_WAIT;
    }
    if (over) {
        snprintf(msg, sizeof(msg), "wp_batch_results: %d grid(s) above the relative tolerance %g after replay", over,
                 B->prm.rel_tol);
        wp_set_error_msg(msg);
        return WP_ERR_NOT_CONVERGED;
    }
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_batch_set_mode(wp_batch* B, int mode, long long tile_cells) {
    if (!B || (mode != WP_BATCH_GRAPH && mode != WP_BATCH_PERSISTENT && mode != WP_BATCH_AUTO) || tile_cells < 0 ||
        tile_cells > (1LL << 30)) {
        wp_set_error_msg("wp_batch_set_mode: mode WP_BATCH_GRAPH, WP_BATCH_PERSISTENT or WP_BATCH_AUTO, "
                         "0 <= tile_cells <= 2^30");
        return WP_ERR_INVALID_ARG;
    }
    wp_mg_pbatch* old = B->pb;
    const long long old_cells = B->tile_cells;
    const bool old_auto = B->tile_auto;
    B->pb = nullptr;
    B->tile_cells = tile_cells;
    B->tile_auto = tile_cells == 0;
    bool pers_ok = true;
    if (mode == WP_BATCH_PERSISTENT || mode == WP_BATCH_AUTO) {
        // checked now, so an unsupported batch fails here and keeps its mode (AUTO: runs as a graph)
        const wp_status st = build_pbatch(B);
        if (st != WP_OK && mode == WP_BATCH_AUTO && st == WP_ERR_UNSUPPORTED) {
            pers_ok = false;
        } else if (st != WP_OK) {
            B->pb = old;
            B->tile_cells = old_cells;
            B->tile_auto = old_auto;
            return st;
        }
    }
    if (old) wp_mg_pbatch_destroy(old);
    B->mode = mode;
    B->run_mode = mode == WP_BATCH_PERSISTENT ? WP_BATCH_PERSISTENT : WP_BATCH_GRAPH;
    B->pers_ok = pers_ok;
    B->graph_ms = 0.f;
    for (float& t : B->tile_ms) t = 0.f;
    destroy_graph(B);
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_batch_get_mode(const wp_batch* B, int* mode, long long* tile_cells,
                                                  float* tuned_ms) {
    if (!B) {
        wp_set_error_msg("wp_batch_get_mode: null handle");
        return WP_ERR_INVALID_ARG;
    }
    if (mode) *mode = B->run_mode;
    if (tile_cells) *tile_cells = B->tile_cells ? B->tile_cells : 32768;
    if (tuned_ms) {
        for (int k = 0; k < kTileN; ++k) tuned_ms[k] = B->tile_ms[k];
        tuned_ms[kTileN] = B->graph_ms;
    }
    return WP_OK;
}

extern "C" CUWHHD_API wp_status wp_batch_profile(wp_batch* B, int enable, double* out, int cap, void* stream) {
    if (!B || cap < 0 || (cap > 0 && !out)) {
        wp_set_error_msg("wp_batch_profile: bad arguments");
        return WP_ERR_INVALID_ARG;
    }
    if (B->run_mode != WP_BATCH_PERSISTENT || !B->pb) {
        wp_set_error_msg("wp_batch_profile: the batch's solves do not run in the persistent kernel");
        return WP_ERR_UNSUPPORTED;
    }
    std::vector<unsigned long long> v(wp_mg_pbatch_prof_slots(), 0ull);
    wp_status st = wp_mg_pbatch_profile(B->pb, enable, v.data(), (cudaStream_t)stream);
    for (int k = 0; k < cap && k < (int)v.size(); ++k) out[k] = (double)v[k];
    return st;
}

extern "C" CUWHHD_API wp_status wp_batch_destroy(wp_batch* B) {
    if (!B) return WP_OK;
    destroy_graph(B);
    if (B->pb) wp_mg_pbatch_destroy(B->pb);
    for (auto& G : B->g) {
        if (G.mg3) wp_mgfrac3d_destroy(G.mg3);
        if (G.mg2) wp_mgfrac2d_destroy(G.mg2);
        if (G.rec3) wp_recover3d_destroy(G.rec3);
        if (G.rec2) wp_recover2d_destroy(G.rec2);
        if (G.b) cudaFree(G.b);
        if (G.p) cudaFree(G.p);
    }
    for (auto& s : B->streams) cudaStreamDestroy(s);
    for (auto& e : B->events) cudaEventDestroy(e);
    if (B->d_max) cudaFree(B->d_max);
    if (B->d_slots) cudaFree((void*)B->d_slots);
    if (B->d_loops) cudaFree((void*)B->d_loops);
    if (B->d_out) cudaFree(B->d_out);
    delete B;
    return WP_OK;
}
