// Autotuner: picks the context's tunables by timing candidates on the caller's own
// workload, then keeps the fastest.  Tunables change speed only, never results (every
// traversal variant and budget makes the same decisions), so tuning is safe to run at
// any time between renders or queries.
//   lux_autotune_trace   ray queries: traversal variant (binary / 4-wide nodes, one
//                        thread per ray / persistent warps) x steps per refill round
//   lux_autotune_render  path tracer: one thread per path vs refilling lanes x steps per
//                        refill round x paths per wavefront batch, then the refilling
//                        kernels' blocks per SM
// Each candidate runs `repeats` times on ctx's stream between CUDA events; its time is
// the fastest repeat.  No reference counterpart (the reference has fixed launch shapes).

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/lux_gpu.h"
#include "lux_internal.h"
#include "pt_scene.h"

namespace {

struct Candidate {
    int variant;
    int budget;
    int batch;
    int blocks = 0;   // refilling kernels' blocks per SM (0: as many as fit)
};

template <typename Run>
int time_candidate(lux_ctx* ctx, int repeats, Run run, float* best_ms) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess)
        return lux::cuda_fail(cudaGetLastError(), "tuning events");
    float best = INFINITY;
    int st = LUX_OK;
    for (int r = 0; r < repeats && !st; ++r) {
        cudaEventRecord(a, ctx->stream);
        st = run();
        cudaEventRecord(b, ctx->stream);
        cudaError_t err = cudaEventSynchronize(b);
        if (!st && err != cudaSuccess) st = lux::cuda_fail(err, "tuning run");
        float ms = 0;
        if (!st) cudaEventElapsedTime(&ms, a, b);
        if (!st) best = std::min(best, ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *best_ms = best;
    return st;
}

int check_error_word(lux_ctx* ctx) {
    int word = 0;
    cudaError_t err = cudaMemcpy(&word, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return lux::cuda_fail(err, "error word read");
    if (word) {
        cudaMemset(ctx->d_error, 0, sizeof(int));
        return lux::fail(LUX_ERR_DEVICE_CHECK, "device check failed during tuning");
    }
    return LUX_OK;
}

void apply(lux_ctx* ctx, const Candidate& c, bool render) {
    ctx->trace_variant = c.variant;
    if (render) {
        ctx->path_budget = c.budget;
        ctx->render_batch = c.batch;
        ctx->refill_blocks = c.blocks;
    } else {
        ctx->trace_budget = c.budget;
    }
}

}  // namespace

extern "C" int lux_autotune_trace(lux_ctx* ctx, lux_bvh* bvh, const float* rays, int32_t n,
                                  lux_tune_result* out) {
    if (!ctx || !bvh || !out || n <= 0 || !rays)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "autotune needs a context, a BVH and rays");
    if (!bvh->has_triangles) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "BVH has no triangles");
    if (cudaError_t err = cudaSetDevice(ctx->device)) return lux::cuda_fail(err, "cudaSetDevice");
    cudaPointerAttributes attr{};
    bool dev = cudaPointerGetAttributes(&attr, rays) == cudaSuccess &&
               (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    if (!dev) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "autotune takes device rays");
    int* hit_id = nullptr;
    float* hit_t = nullptr;
    cudaError_t err = cudaMalloc(&hit_id, sizeof(int) * size_t(n));
    if (err == cudaSuccess) err = cudaMalloc(&hit_t, sizeof(float) * size_t(n));
    if (err != cudaSuccess) {
        cudaFree(hit_id);
        return lux::fail(LUX_ERR_OUT_OF_MEMORY, "autotune buffers");
    }
    const Candidate before{ctx->trace_variant, ctx->trace_budget, ctx->render_batch};
    std::vector<Candidate> cands;
    cands.push_back(before);
    for (int v : {lux::kTraceStatic, lux::kTraceWide}) cands.push_back({v, 16, 0});
    for (int v : {lux::kTracePersistent, lux::kTraceWidePersistent})
        for (int b : {8, 16, 32, 64}) cands.push_back({v, b, 0});
    int st = LUX_OK;
    float best_ms = INFINITY, default_ms = INFINITY;
    Candidate best = before;
    for (size_t i = 0; i < cands.size() && !st; ++i) {
        apply(ctx, cands[i], false);
        float ms = 0;
        st = time_candidate(ctx, 3, [&] {
            return lux::trace_closest(ctx, bvh, rays, n, hit_id, hit_t);
        }, &ms);
        if (!st) st = check_error_word(ctx);
        if (st) break;
        if (i == 0) default_ms = ms;
        if (ms < best_ms) {
            best_ms = ms;
            best = cands[i];
        }
    }
    cudaFree(hit_id);
    cudaFree(hit_t);
    apply(ctx, st ? before : best, false);
    if (st) return st;
    out->trace_variant = best.variant;
    out->budget = best.budget;
    out->render_batch = 0;
    out->refill_blocks = 0;
    out->best_ms = best_ms;
    out->default_ms = default_ms;
    out->candidates = static_cast<int32_t>(cands.size());
    return LUX_OK;
}

extern "C" int lux_autotune_render(lux_ctx* ctx, const lux_scene* scene,
                                   const lux_render_request* probe, lux_tune_result* out) {
    if (!ctx || !scene || !probe || !out)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "autotune needs a context, a scene and a probe");
    if (probe->width <= 0 || probe->height <= 0 || probe->spp <= 0 || probe->max_depth < 0)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "probe request needs a non-empty film");
    if (cudaError_t err = cudaSetDevice(ctx->device)) return lux::cuda_fail(err, "cudaSetDevice");
    const size_t pixels = static_cast<size_t>(probe->width) * probe->height;
    const long long paths = static_cast<long long>(pixels) * probe->spp;
    float* film = nullptr;
    if (cudaMalloc(&film, sizeof(float) * 3 * pixels) != cudaSuccess) {
        cudaGetLastError();
        return lux::fail(LUX_ERR_OUT_OF_MEMORY, "autotune film");
    }
    const Candidate before{ctx->trace_variant, ctx->path_budget, ctx->render_batch,
                           ctx->refill_blocks};
    std::vector<Candidate> cands;
    cands.push_back(before);
    std::vector<int> batches;
    for (long long b : {1ll << 20, 1ll << 21, 1ll << 22, 1ll << 23})
        if (b <= std::max<long long>(paths, 1ll << 20)) batches.push_back(static_cast<int>(b));
    for (int batch : batches) {
        cands.push_back({lux::kTraceStatic, before.budget, batch});
        for (int b : {8, 16, 32, 64}) cands.push_back({lux::kTraceAuto, b, batch});
    }
    int st = LUX_OK;
    float best_ms = INFINITY, default_ms = INFINITY;
    Candidate best = before;
    auto run = [&](const Candidate& c, float* ms) {
        apply(ctx, c, true);
        int s2 = time_candidate(ctx, 2, [&] { return lux::render(ctx, scene, *probe, film, false); },
                                ms);
        if (!s2) s2 = check_error_word(ctx);
        return s2;
    };
    for (size_t i = 0; i < cands.size() && !st; ++i) {
        float ms = 0;
        st = run(cands[i], &ms);
        if (st) break;
        if (i == 0) default_ms = ms;
        if (ms < best_ms) {
            best_ms = ms;
            best = cands[i];
        }
    }
    // Second stage, refilling lanes only: fewer resident blocks per SM than fit (fewer
    // warps, more cache and shared bandwidth each).
    int tried = static_cast<int>(cands.size());
    if (!st && best.variant != lux::kTraceStatic) {
        for (int blocks : {1, 2}) {
            Candidate c = best;
            c.blocks = blocks;
            float ms = 0;
            st = run(c, &ms);
            ++tried;
            if (st) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
    }
    cudaFree(film);
    apply(ctx, st ? before : best, true);
    if (st) return st;
    out->trace_variant = best.variant;
    out->budget = best.budget;
    out->render_batch = best.batch;
    out->best_ms = best_ms;
    out->default_ms = default_ms;
    out->candidates = tried;
    out->refill_blocks = best.blocks;
    return LUX_OK;
}
