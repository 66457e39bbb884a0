// Single-request wavefront path tracer for sm_100a.
//
// A render is a sequence of batches; a batch holds (pixel range) x (sample range) paths,
// pixel-major, so a pixel's samples are adjacent.  Per bounce d:
//   k_extend   closest hit through TLAS -> BLAS for every path in ray queue d; misses
//              add environment radiance; hits are appended to one of five material
//              queues (warp-aggregated appends)
//   k_shade    all material queues in one launch (warps stay on one material): emission
//              with MIS, pass-through, NEE light sample -> shadow queue, BSDF sample,
//              Russian roulette -> ray queue d+1
//   k_shadow   shadow rays through pass-through surfaces; adds the NEE contribution
// then k_flush adds each pixel's sample radiances to the film in sample order, which is
// the reference CPU tracer's float accumulation order (cpu_path_tracer.cpp:543-558).
//
// Reference counterparts (src/): integrator/wavefront_kernels.cu:234-715,
// integrator/wavefront_scheduler.cu:73-131.  Queue sizes live on the device; kernels
// use grid-stride loops over them, so no bounce waits for the host.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>

#include "../../include/lux_gpu.h"
#include "pt_kernels.cuh"
#include "pt_scene.h"

namespace lux {
namespace pt {
namespace {

constexpr int kSlots = 9;  // per-bounce counters: ray, 5 material queues, shadow, extend and
                           // shadow cursors

// Depth slots of the queue counters: every max_depth the API accepts (0..1000), so the
// counters are allocated once per runtime and a deeper request never reallocates.
constexpr int kMaxDepthSlots = 1000 + 2;

// Batches of one render run on kRenderLanes lanes in turn, each with its own path pool,
// counters and stream (lane 0 the context's, the others the runtime's own): while one
// batch's last bounces drain (few paths, long walks, most SMs idle) the next batch's
// first bounces fill the GPU.  Each batch's film accumulation waits for the previous
// batch's, so the film sums in the same sample order as with one lane.
#ifndef LUX_RENDER_LANES
#define LUX_RENDER_LANES 4
#endif
constexpr int kRenderLanes = LUX_RENDER_LANES;

struct Runtime {
    PathPool pool[kRenderLanes];
    int* counts[kRenderLanes] = {};      // kMaxDepthSlots * kSlots per lane
    unsigned long long* rays = nullptr;  // [0] camera + extension, [1] shadow segments
    long long last_counts[2] = {0, 0};
    int lanes = 0;                       // lanes allocated
    cudaStream_t stream[kRenderLanes] = {};   // lanes 1.. (lane 0 runs on the context's)
    cudaEvent_t ev_setup = nullptr;
    cudaEvent_t ev_end[kRenderLanes] = {};
    cudaEvent_t ev_flush[kRenderLanes] = {};
};

struct Batch {
    int pixel0, pixels;     // pixel range
    int sample0, samples;   // sample range (request-relative)
    CameraParams cam;
};

__global__ void __launch_bounds__(kThreads) k_camera(PathPool rt, int* counts, SceneView sc,
                                                     Batch b) {
    int n = b.pixels * b.samples;
    if (blockIdx.x == 0 && threadIdx.x == 0) counts[0] = n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        init_path(rt, sc.camera, i, b.pixel0 + i / b.samples, b.sample0 + i % b.samples, b.cam);
        rt.qray[0][i] = i;
    }
}

__global__ void __launch_bounds__(kThreads) k_extend(PathPool rt, int* counts, SceneView sc,
                                                     int sampler, int depth, int* error) {
    int n = counts[depth * kSlots];
    int* mat_counts = counts + depth * kSlots + 1;
    const int* q = rt.qray[depth & 1];
    int stride = gridDim.x * blockDim.x;
    int rounds = (n + stride - 1) / stride;
    for (int r = 0; r < rounds; ++r) {
        int i = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
        bool active = i < n;
        int p = active ? q[i] : 0;
        int cls = active ? extend_path(rt, sc, sampler, p, error) : -1;
        bool hit = cls >= 0;
        int slot = append(mat_counts, hit ? cls : 0, hit);
        if (hit) rt.qmat[cls * rt.capacity + slot] = p;
    }
}

// k_extend with refilling lanes (refill_walks); the cursor is the bounce's spare slot.
// Three resident blocks per SM (at most 80 registers, 64 bytes of spills) rather than the
// two that 103 registers allow: latency-bound walks gain more from the extra warps (heavy
// scene 1330 -> 1507 Mrays/s on one B200).
__global__ void __launch_bounds__(kThreads, 3) k_extend_refill(PathPool rt, int* counts,
                                                            SceneView sc, int sampler, int depth,
                                                            int budget, int* error) {
    int* c = counts + depth * kSlots;
    int* mat_counts = c + 1;
    refill_walks(
        rt, rt.qray[depth & 1], c[0], c + 7, budget, error, [](int) { return 0; },
        [&](int) -> const SceneView& { return sc; },
        [&](int p, int, const SceneHit& h) {
            const int cls = p >= 0 ? extend_finish(rt, sc, sampler, p, h) : -1;
            const bool hit = cls >= 0;
            const int slot = append(mat_counts, hit ? cls : 0, hit);
            if (hit) rt.qmat[cls * rt.capacity + slot] = p;
        });
}

// Three resident blocks per SM (at most 80 registers) as k_extend_refill.
#ifndef LUX_SHADE_BLOCKS
#define LUX_SHADE_BLOCKS 3
#endif
__global__ void __launch_bounds__(kThreads, LUX_SHADE_BLOCKS) k_shade(PathPool rt, int* counts, SceneView sc,
                                                    int sampler, int depth, int max_depth) {
    const int* mc = counts + depth * kSlots + 1;
    int* next_count = counts + (depth + 1) * kSlots;
    int* shadow_count = counts + depth * kSlots + 6;
    int c[kClasses];
    int total = 0;
    for (int k = 0; k < kClasses; ++k) {
        c[k] = mc[k];
        total += c[k];
    }
    int* qnext = rt.qray[(depth + 1) & 1];
    int stride = gridDim.x * blockDim.x;
    int rounds = (total + stride - 1) / stride;
    for (int r = 0; r < rounds; ++r) {
        int i = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
        bool active = i < total;
        int cls = 0, j = i;
        while (cls < kClasses - 1 && j >= c[cls]) j -= c[cls++];
        int p = active ? rt.qmat[cls * rt.capacity + j] : 0;
        ShadeOut o;
        if (active) o = shade_path(rt, sc, sampler, max_depth, p);
        int slot = append(shadow_count, 0, o.shadow);
        if (o.shadow) rt.qshadow[slot] = p;
        slot = append(next_count, 0, o.spawn);
        if (o.spawn) qnext[slot] = p;
    }
}

__global__ void __launch_bounds__(kThreads) k_shadow(PathPool rt, int* counts,
                                                     unsigned long long* rays, SceneView sc,
                                                     int depth, int* error) {
    int n = counts[depth * kSlots + 6];
    unsigned long long segments = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        shadow_path(rt, sc, rt.qshadow[i], error, segments);
    warp_add(rays + 1, segments);
}

// k_shadow with refilling lanes (refill_shadows); the cursor is the bounce's slot 8.
__global__ void __launch_bounds__(kThreads, 3) k_shadow_refill(PathPool rt, int* counts,
                                                            unsigned long long* rays,
                                                            SceneView sc, int depth, int budget,
                                                            int* error) {
    int* c = counts + depth * kSlots;
    unsigned long long segments = 0;
    refill_shadows(
        rt, rt.qshadow, c[6], c + 8, budget, error, [](int) { return 0; },
        [&](int) -> const SceneView& { return sc; },
        [&](int p, f3 v) { add_radiance(rt, p, v); }, segments);
    warp_add(rays + 1, segments);
}

// The bounce kernels with the debug images (one path per thread, closest-hit shadow
// segments, as the classification needs the blocking hit).
__global__ void __launch_bounds__(kThreads) k_extend_aov(PathPool rt, int* counts, SceneView sc,
                                                         int sampler, int depth, int* error,
                                                         DebugTargets aov) {
    int n = counts[depth * kSlots];
    int* mat_counts = counts + depth * kSlots + 1;
    const int* q = rt.qray[depth & 1];
    int stride = gridDim.x * blockDim.x;
    int rounds = (n + stride - 1) / stride;
    for (int r = 0; r < rounds; ++r) {
        int i = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
        bool active = i < n;
        int p = active ? q[i] : 0;
        int cls = -1;
        if (active) {
            const float4 a = rt.ray_o[p], b = rt.ray_d[p];
            SceneHit h;
            if (aov.walk_counts) {
                WalkCounts wc;
                h = scene_closest<true>(sc, xyz(a), xyz(b), a.w, b.w, -1, error, &wc);
                atomicAdd(aov.walk_counts, wc.boxes);
                atomicAdd(aov.walk_counts + 1, wc.tris);
                atomicAdd(aov.walk_counts + 2, wc.instances);
            } else {
                h = scene_closest(sc, xyz(a), xyz(b), a.w, b.w, -1, error);
            }
            if (depth == 0) aov_primary(rt, sc, p, h, aov);
            cls = extend_finish(rt, sc, sampler, p, h);
        }
        bool hit = cls >= 0;
        int slot = append(mat_counts, hit ? cls : 0, hit);
        if (hit) rt.qmat[cls * rt.capacity + slot] = p;
    }
}

__global__ void __launch_bounds__(kThreads) k_shade_aov(PathPool rt, int* counts, SceneView sc,
                                                        int sampler, int depth, int max_depth,
                                                        DebugTargets aov) {
    const int* mc = counts + depth * kSlots + 1;
    int* next_count = counts + (depth + 1) * kSlots;
    int* shadow_count = counts + depth * kSlots + 6;
    int total = 0;
    for (int k = 0; k < kClasses; ++k) total += mc[k];
    int* qnext = rt.qray[(depth + 1) & 1];
    int stride = gridDim.x * blockDim.x;
    int rounds = (total + stride - 1) / stride;
    for (int r = 0; r < rounds; ++r) {
        int i = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
        bool active = i < total;
        int cls = 0, j = i;
        while (cls < kClasses - 1 && j >= mc[cls]) j -= mc[cls++];
        int p = active ? rt.qmat[cls * rt.capacity + j] : 0;
        ShadeOut o;
        if (active) o = shade_path<true>(rt, sc, sampler, max_depth, p, aov);
        int slot = append(shadow_count, 0, o.shadow);
        if (o.shadow) rt.qshadow[slot] = p;
        slot = append(next_count, 0, o.spawn);
        if (o.spawn) qnext[slot] = p;
    }
}

__global__ void __launch_bounds__(kThreads) k_shadow_aov(PathPool rt, int* counts,
                                                         unsigned long long* rays, SceneView sc,
                                                         int depth, int* error, DebugTargets aov) {
    int n = counts[depth * kSlots + 6];
    unsigned long long segments = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        shadow_path<true>(rt, sc, rt.qshadow[i], error, segments, aov);
    warp_add(rays + 1, segments);
}

// Per-pixel film accumulation in sample order; or every sample's radiance.
__global__ void __launch_bounds__(kThreads) k_flush(PathPool rt, Batch b, float* film,
                                                    float* samples, int spp) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < b.pixels; j += gridDim.x * blockDim.x) {
        int pixel = b.pixel0 + j;
        if (samples) {
            for (int s = 0; s < b.samples; ++s) {
                float4 r = rt.rad[j * b.samples + s];
                size_t o = (static_cast<size_t>(pixel) * spp + b.sample0 + s) * 3;
                samples[o] = r.x;
                samples[o + 1] = r.y;
                samples[o + 2] = r.z;
            }
        } else {
            float x = film[3 * size_t(pixel)], y = film[3 * size_t(pixel) + 1],
                  z = film[3 * size_t(pixel) + 2];
            for (int s = 0; s < b.samples; ++s) {
                float4 r = rt.rad[j * b.samples + s];
                x = add(x, r.x);
                y = add(y, r.y);
                z = add(z, r.z);
            }
            film[3 * size_t(pixel)] = x;
            film[3 * size_t(pixel) + 1] = y;
            film[3 * size_t(pixel) + 2] = z;
        }
    }
}

// One light selection per thread at a given position (sample_scene_light + light_pmf).
__global__ void k_select_lights(SceneView sc, int sampler, const float* positions,
                                const float* select_u, int n, int32_t* light_index, float* pmf,
                                float* eval_pmf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const f3 p = make_f3(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
    float selected = 0;
    const int index = select_light(sc, sampler, p, select_u[i], selected);
    light_index[i] = index;
    pmf[i] = selected;
    eval_pmf[i] = index >= 0 ? light_pmf(sc, sampler, p, index) : 0.0f;
}

__global__ void k_count_rays(const int* counts, unsigned long long* rays, int depth_slots) {
    unsigned long long total = 0;
    for (int d = 0; d < depth_slots; ++d) total += static_cast<unsigned>(counts[d * kSlots]);
    atomicAdd(rays, total);
}

Runtime* runtime_of(lux_ctx* ctx) { return static_cast<Runtime*>(ctx->render_runtime); }

void runtime_release(Runtime* rt) {
    for (int l = 0; l < kRenderLanes; ++l) {
        path_pool_free(rt->pool[l]);
        if (rt->counts[l]) cudaFree(rt->counts[l]);
    }
    if (rt->rays) cudaFree(rt->rays);
    if (rt->ev_setup) cudaEventDestroy(rt->ev_setup);
    for (int l = 0; l < kRenderLanes; ++l) {
        if (rt->ev_end[l]) cudaEventDestroy(rt->ev_end[l]);
        if (rt->ev_flush[l]) cudaEventDestroy(rt->ev_flush[l]);
        if (rt->stream[l]) cudaStreamDestroy(rt->stream[l]);
    }
    long long keep[2] = {rt->last_counts[0], rt->last_counts[1]};
    *rt = Runtime{};
    rt->last_counts[0] = keep[0];
    rt->last_counts[1] = keep[1];
}

}  // namespace

void path_pool_free(PathPool& p) {
    void* ptrs[] = {p.thr_eta, p.rad, p.prev, p.meta, p.rng, p.ray_o, p.ray_d, p.hit, p.sh_o,
                    p.sh_d, p.sh_c, p.sh_t, p.qray[0], p.qray[1], p.qmat, p.qshadow};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    p = PathPool{};
}

// Shared by the server: device buffers of a path pool of `capacity` paths.
int path_pool_alloc(PathPool& p, int capacity) {
    size_t c = static_cast<size_t>(capacity);
    struct Req {
        void** ptr;
        size_t bytes;
    } reqs[] = {
        {reinterpret_cast<void**>(&p.thr_eta), 16 * c}, {reinterpret_cast<void**>(&p.rad), 16 * c},
        {reinterpret_cast<void**>(&p.prev), 16 * c}, {reinterpret_cast<void**>(&p.meta), 16 * c},
        {reinterpret_cast<void**>(&p.rng), 16 * c}, {reinterpret_cast<void**>(&p.ray_o), 16 * c},
        {reinterpret_cast<void**>(&p.ray_d), 16 * c}, {reinterpret_cast<void**>(&p.hit), 16 * c},
        {reinterpret_cast<void**>(&p.sh_o), 16 * c}, {reinterpret_cast<void**>(&p.sh_d), 16 * c},
        {reinterpret_cast<void**>(&p.sh_c), 16 * c}, {reinterpret_cast<void**>(&p.sh_t), 16 * c},
        {reinterpret_cast<void**>(&p.qray[0]), 4 * c}, {reinterpret_cast<void**>(&p.qray[1]), 4 * c},
        {reinterpret_cast<void**>(&p.qmat), 4 * c * kClasses},
        {reinterpret_cast<void**>(&p.qshadow), 4 * c},
    };
    for (auto& r : reqs) {
        cudaError_t err = cudaMalloc(r.ptr, r.bytes);
        if (err != cudaSuccess) {
            cudaGetLastError();
            return fail(LUX_ERR_OUT_OF_MEMORY, "path pool allocation failed");
        }
    }
    p.capacity = capacity;
    return LUX_OK;
}

namespace {

// Grows the path pools to at least `capacity` paths and `lanes` lanes (never shrinks
// them); the counters are allocated once.  Only a larger batch than any before it (or a
// first render with two lanes) reallocates, so a stream of renders of mixed depth and size
// sized for its largest batch allocates nothing.
int runtime_reserve(lux_ctx* ctx, int capacity, int max_depth, int lanes) {
    Runtime* rt = runtime_of(ctx);
    if (!rt) {
        rt = new (std::nothrow) Runtime();
        if (!rt) return fail(LUX_ERR_OUT_OF_MEMORY, "runtime allocation failed");
        ctx->render_runtime = rt;
    }
    if (max_depth + 2 > kMaxDepthSlots)
        return fail(LUX_ERR_INVALID_ARGUMENT, "max_depth must be in 0..1000");
    if (rt->pool[0].capacity >= capacity && rt->lanes >= lanes && rt->rays) return LUX_OK;
    lanes = std::max(lanes, rt->lanes);
    cudaStreamSynchronize(ctx->stream);
    for (int l = 1; l < kRenderLanes; ++l)
        if (rt->stream[l]) cudaStreamSynchronize(rt->stream[l]);
    runtime_release(rt);
    int st = LUX_OK;
    cudaError_t err = cudaSuccess;
    for (int l = 0; l < lanes && !st && err == cudaSuccess; ++l) {
        st = path_pool_alloc(rt->pool[l], capacity);
        if (!st) err = cudaMalloc(&rt->counts[l], sizeof(int) * kSlots * kMaxDepthSlots);
    }
    if (!st && err == cudaSuccess) err = cudaMalloc(&rt->rays, 16);
    if (!st && err == cudaSuccess && lanes > 1) {
        err = cudaEventCreateWithFlags(&rt->ev_setup, cudaEventDisableTiming);
        for (int l = 0; l < lanes && err == cudaSuccess; ++l) {
            if (l > 0) err = cudaStreamCreateWithFlags(&rt->stream[l], cudaStreamNonBlocking);
            if (err == cudaSuccess) err = cudaEventCreateWithFlags(&rt->ev_end[l], cudaEventDisableTiming);
            if (err == cudaSuccess) err = cudaEventCreateWithFlags(&rt->ev_flush[l], cudaEventDisableTiming);
        }
    }
    if (!st && err != cudaSuccess) {
        cudaGetLastError();
        st = fail(LUX_ERR_OUT_OF_MEMORY, "wavefront runtime allocation failed");
    }
    if (st) {
        runtime_release(rt);
        return st;
    }
    rt->lanes = lanes;
    return LUX_OK;
}

}  // namespace
}  // namespace pt

void render_runtime_free(lux_ctx* ctx) {
    pt::Runtime* rt = pt::runtime_of(ctx);
    if (!rt) return;
    pt::runtime_release(rt);
    delete rt;
    ctx->render_runtime = nullptr;
}

int select_lights(lux_ctx* ctx, const lux_scene* scene, int sampler, const float* positions,
                  const float* select_u, int n, int32_t* light_index, float* pmf,
                  float* eval_pmf) {
    pt::k_select_lights<<<(n + pt::kThreads - 1) / pt::kThreads, pt::kThreads, 0, ctx->stream>>>(
        scene->view, sampler, positions, select_u, n, light_index, pmf, eval_pmf);
    ctx->launches += 1;
    cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? LUX_OK : cuda_fail(err, "light selection");
}

int render_ray_counts(lux_ctx* ctx, int64_t* counts) {
    pt::Runtime* rt = pt::runtime_of(ctx);
    counts[0] = rt ? rt->last_counts[0] : 0;
    counts[1] = rt ? rt->last_counts[1] : 0;
    return LUX_OK;
}

int render(lux_ctx* ctx, const lux_scene* scene, const lux_render_request& req, float* out,
           bool per_sample, float* aov_shadow, float* aov_ng, float* aov_ns,
           lux_path_log_record* log, unsigned long long* log_count, long long log_capacity,
           unsigned long long* walk_counts) {
    using namespace pt;
    DebugTargets aov;
    aov.shadow = aov_shadow;
    aov.ng = aov_ng;
    aov.ns = aov_ns;
    aov.log = log_capacity > 0 ? log : nullptr;
    aov.log_count = log_count;
    aov.log_capacity = aov.log ? log_capacity : 0;
    aov.sample_offset = req.sample_offset;
    aov.walk_counts = walk_counts;
    const bool with_aov = aov_shadow || aov_ng || aov_ns || log_count || walk_counts;
    const int pixels = req.width * req.height;
    const long long total_paths = static_cast<long long>(pixels) * req.spp;
    // Batch: whole pixels' sample ranges, at most ctx->render_batch paths.
    int batch_cap = std::max(1, ctx->render_batch);
    int samples_per_batch = static_cast<int>(
        std::min<long long>(req.spp, std::max(1, batch_cap / std::max(pixels, 1))));
    int pixels_per_batch = samples_per_batch > 1 || samples_per_batch >= req.spp
                               ? pixels : std::min(pixels, batch_cap);
    int capacity = static_cast<int>(std::min<long long>(
        total_paths, static_cast<long long>(pixels_per_batch) * samples_per_batch));
    // Up to kRenderLanes lanes when there is more than one batch; one for the debug
    // outputs, whose atomically indexed records and sums keep the one-lane order.
    const long long batches =
        ((req.spp + samples_per_batch - 1) / samples_per_batch) *
        static_cast<long long>((pixels + pixels_per_batch - 1) / std::max(pixels_per_batch, 1));
    const int lanes =
        !with_aov && batches > 1 ? static_cast<int>(std::min<long long>(kRenderLanes, batches)) : 1;
    int st = runtime_reserve(ctx, std::max(capacity, 1), req.max_depth, lanes);
    if (st) return st;
    Runtime& rt = *runtime_of(ctx);
    const SceneView& sc = scene->view;
    cudaStream_t s0 = ctx->stream;
    cudaStream_t s = s0;
    int grid = ctx->sm_count * 8;
    // Persistent grids of the refilling kernels: blocks per SM up to what fits, or the
    // context's LUX_OPT_REFILL_BLOCKS when it asks for fewer.
    const int refill_fit = occupancy_blocks(ctx, kOccExtendRefill, k_extend_refill, kThreads);
    const int shadow_fit = occupancy_blocks(ctx, kOccShadowRefill, k_shadow_refill, kThreads);
    const int refill_grid =
        ctx->sm_count * (ctx->refill_blocks > 0 ? std::min(ctx->refill_blocks, refill_fit)
                                                : refill_fit);
    const int shadow_grid =
        ctx->sm_count * (ctx->refill_blocks > 0 ? std::min(ctx->refill_blocks, shadow_fit)
                                                : shadow_fit);
    cudaError_t err = cudaMemsetAsync(rt.rays, 0, 16, s);
    if (!per_sample && err == cudaSuccess)
        err = cudaMemsetAsync(out, 0, sizeof(float) * 3 * size_t(pixels), s);
    for (float* image : {aov_shadow, aov_ng, aov_ns})
        if (image && err == cudaSuccess)
            err = cudaMemsetAsync(image, 0, sizeof(float) * 3 * size_t(pixels), s);
    if (log_count && err == cudaSuccess)
        err = cudaMemsetAsync(log_count, 0, sizeof(unsigned long long), s);
    if (walk_counts && err == cudaSuccess)
        err = cudaMemsetAsync(walk_counts, 0, 3 * sizeof(unsigned long long), s);
    if (lanes > 1 && err == cudaSuccess) {
        // The other lanes start after the setup.
        err = cudaEventRecord(rt.ev_setup, s0);
        for (int l = 1; l < lanes && err == cudaSuccess; ++l)
            err = cudaStreamWaitEvent(rt.stream[l], rt.ev_setup, 0);
    }
    if (err != cudaSuccess) return cuda_fail(err, "render setup");
    // A failure after the second lane started waits for that lane before returning, so
    // no kernel of this render is left running on the runtime's buffers.
    auto lane_fail = [&](cudaError_t e, const char* what) {
        for (int l = 1; l < lanes; ++l) cudaStreamSynchronize(rt.stream[l]);
        return cuda_fail(e, what);
    };
    long long k = 0;   // batch index
    for (int sa = 0; sa < req.spp; sa += samples_per_batch) {
        int ns = std::min(samples_per_batch, req.spp - sa);
        for (int p0 = 0; p0 < pixels; p0 += pixels_per_batch, ++k) {
            const int lane = static_cast<int>(k % lanes);
            s = lane ? rt.stream[lane] : s0;
            const PathPool& pool = rt.pool[lane];
            int* counts = rt.counts[lane];
            Batch b;
            b.pixel0 = p0;
            b.pixels = std::min(pixels_per_batch, pixels - p0);
            b.sample0 = sa;
            b.samples = ns;
            b.cam = CameraParams{req.width, req.height, req.seed, req.frame_index, req.sample_offset};
            err = cudaMemsetAsync(counts, 0, sizeof(int) * kSlots * (req.max_depth + 2), s);
            if (err != cudaSuccess) return lane_fail(err, "counter reset");
            k_camera<<<grid, kThreads, 0, s>>>(pool, counts, sc, b);
            ctx->launches += 1;
            for (int d = 0; d <= req.max_depth; ++d) {
                if (with_aov) {
                    k_extend_aov<<<grid, kThreads, 0, s>>>(pool, counts, sc,
                                                           req.light_sampler, d, ctx->d_error, aov);
                    k_shade_aov<<<grid, kThreads, 0, s>>>(pool, counts, sc,
                                                          req.light_sampler, d, req.max_depth, aov);
                    k_shadow_aov<<<grid, kThreads, 0, s>>>(pool, counts, rt.rays, sc, d,
                                                           ctx->d_error, aov);
                    ctx->launches += 3;
                    continue;
                }
                if (ctx->trace_variant == kTraceStatic) {
                    k_extend<<<grid, kThreads, 0, s>>>(pool, counts, sc, req.light_sampler,
                                                       d, ctx->d_error);
                } else {
                    k_extend_refill<<<refill_grid, kThreads, 0, s>>>(
                        pool, counts, sc, req.light_sampler, d, ctx->path_budget,
                        ctx->d_error);
                }
                k_shade<<<grid, kThreads, 0, s>>>(pool, counts, sc, req.light_sampler, d,
                                                  req.max_depth);
                if (ctx->trace_variant == kTraceStatic) {
                    k_shadow<<<grid, kThreads, 0, s>>>(pool, counts, rt.rays, sc, d,
                                                       ctx->d_error);
                } else {
                    k_shadow_refill<<<shadow_grid, kThreads, 0, s>>>(
                        pool, counts, rt.rays, sc, d, ctx->path_budget, ctx->d_error);
                }
                ctx->launches += 3;
            }
            k_count_rays<<<1, 1, 0, s>>>(counts, rt.rays, req.max_depth + 1);
            int fgrid = std::max(1, std::min(grid, (b.pixels + kThreads - 1) / kThreads));
            // The film takes the batches in order: this flush follows the previous one.
            if (lanes > 1 && k > 0)
                err = cudaStreamWaitEvent(s, rt.ev_flush[(lane + lanes - 1) % lanes], 0);
            k_flush<<<fgrid, kThreads, 0, s>>>(pool, b, per_sample ? nullptr : out,
                                               per_sample ? out : nullptr, req.spp);
            ctx->launches += 2;
            if (lanes > 1 && err == cudaSuccess) err = cudaEventRecord(rt.ev_flush[lane], s);
            if (err == cudaSuccess) err = cudaGetLastError();
            if (err != cudaSuccess) return lane_fail(err, "render launch");
        }
    }
    for (int l = 1; l < lanes; ++l) {
        // The caller's stream waits for the other lanes.
        err = cudaEventRecord(rt.ev_end[l], rt.stream[l]);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(s0, rt.ev_end[l], 0);
        if (err != cudaSuccess) return cuda_fail(err, "render lanes");
    }
    unsigned long long counts[2];
    err = cudaMemcpyAsync(counts, rt.rays, 16, cudaMemcpyDeviceToHost, s0);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s0);
    if (err != cudaSuccess) return cuda_fail(err, "render");
    rt.last_counts[0] = static_cast<long long>(counts[0]);
    rt.last_counts[1] = static_cast<long long>(counts[1]);
    return LUX_OK;
}

}  // namespace lux
