// extern "C" boundary of liblux_gpu.so (declared in include/lux_gpu.h).
//
// Responsibilities: argument validation, status codes and the thread-local error text,
// host/device pointer classification with staging of host buffers, and the device
// error word that bounded kernel loops report through.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/lux_gpu.h"
#include "lux_internal.h"
#include "pt_scene.h"

namespace {

thread_local std::string g_error;

// Where an argument lives, seen from a context on `device`: host memory (pageable or
// pinned), memory the device can use directly (its own device memory, or managed
// memory), or device memory of another GPU, which no call accepts (without peer access a
// kernel on this device would fault on it).
enum class PtrKind { kHost, kDevice, kOtherDevice };

PtrKind pointer_kind(const void* p, int device) {
    if (!p) return PtrKind::kHost;
    cudaPointerAttributes attr;
    cudaError_t err = cudaPointerGetAttributes(&attr, p);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return PtrKind::kHost;
    }
    if (attr.type == cudaMemoryTypeManaged) return PtrKind::kDevice;
    if (attr.type == cudaMemoryTypeDevice)
        return attr.device == device ? PtrKind::kDevice : PtrKind::kOtherDevice;
    return PtrKind::kHost;
}

bool is_device_pointer(const void* p, int device) {
    return pointer_kind(p, device) == PtrKind::kDevice;
}

// Carves device staging regions for host arguments out of the context's staging buffer.
struct Staging {
    lux_ctx* ctx;
    struct Item {
        const void* host_in;   // copy host -> device before the work
        void* host_out;        // copy device -> host after the work
        size_t bytes;
        size_t offset;
        void** device;
    };
    std::vector<Item> items;
    size_t total = 0;
    bool foreign = false;   // an argument is device memory of another GPU

    explicit Staging(lux_ctx* c) : ctx(c) {}

    // in: the argument is read by the device; out: it is written by the device.
    void add(const void* arg, size_t bytes, bool in, bool out, void** device) {
        if (!arg || bytes == 0) {
            *device = const_cast<void*>(arg);
            return;
        }
        PtrKind kind = pointer_kind(arg, ctx->device);
        if (kind == PtrKind::kOtherDevice) {
            foreign = true;
            *device = nullptr;
            return;
        }
        if (kind == PtrKind::kDevice) {
            *device = const_cast<void*>(arg);
            return;
        }
        Item it{in ? arg : nullptr, out ? const_cast<void*>(arg) : nullptr, bytes, total, device};
        total += (bytes + 255) & ~size_t(255);
        items.push_back(it);
    }

    bool has_host_output() const {
        for (const Item& it : items)
            if (it.host_out) return true;
        return false;
    }

    int begin() {
        if (foreign)
            return lux::fail(LUX_ERR_INVALID_ARGUMENT,
                             "a device pointer belongs to another GPU than the context's");
        if (items.empty()) return LUX_OK;
        if (total > ctx->staging_bytes) {
            if (ctx->staging) {
                cudaStreamSynchronize(ctx->stream);
                cudaFree(ctx->staging);
                ctx->staging = nullptr;
                ctx->staging_bytes = 0;
            }
            cudaError_t err = cudaMalloc(&ctx->staging, total);
            if (err != cudaSuccess) {
                cudaGetLastError();
                return lux::fail(LUX_ERR_OUT_OF_MEMORY, "staging allocation failed");
            }
            ctx->staging_bytes = total;
        }
        char* base = static_cast<char*>(ctx->staging);
        for (Item& it : items) {
            *it.device = base + it.offset;
            if (it.host_in) {
                cudaError_t err = cudaMemcpyAsync(base + it.offset, it.host_in, it.bytes,
                                                  cudaMemcpyHostToDevice, ctx->stream);
                if (err != cudaSuccess) return lux::cuda_fail(err, "host to device copy");
            }
        }
        return LUX_OK;
    }

    int finish() {
        char* base = static_cast<char*>(ctx->staging);
        for (Item& it : items) {
            if (!it.host_out) continue;
            cudaError_t err = cudaMemcpyAsync(it.host_out, base + it.offset, it.bytes,
                                              cudaMemcpyDeviceToHost, ctx->stream);
            if (err != cudaSuccess) return lux::cuda_fail(err, "device to host copy");
        }
        return LUX_OK;
    }
};

int check_ctx(lux_ctx* ctx) {
    if (!ctx) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null context");
    cudaError_t err = cudaSetDevice(ctx->device);
    return lux::cuda_fail(err, "cudaSetDevice");
}

// Waits for the stream, then reports (and clears) the device error word.
int sync_and_check(lux_ctx* ctx) {
    cudaError_t err = cudaStreamSynchronize(ctx->stream);
    if (err != cudaSuccess) return lux::cuda_fail(err, "stream synchronize");
    int word = 0;
    err = cudaMemcpy(&word, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return lux::cuda_fail(err, "error word read");
    if (word) {
        cudaMemset(ctx->d_error, 0, sizeof(int));
        std::string what;
        if (word & lux::kErrClimbBound) what += " bottom-up level bound exceeded;";
        if (word & lux::kErrStackOverflow) what += " traversal stack overflow;";
        if (word & lux::kErrLoopBound) what += " bounded loop exhausted;";
        if (word & lux::kErrQueueOverflow) {
            return lux::fail(LUX_ERR_QUEUE_OVERFLOW, "device check:" + what + " queue overflow");
        }
        return lux::fail(LUX_ERR_DEVICE_CHECK, "device check:" + what);
    }
    return LUX_OK;
}

int finish_call(lux_ctx* ctx, Staging& staging) {
    int st = staging.finish();
    if (st) return st;
    if (staging.has_host_output()) return sync_and_check(ctx);
    return lux::cuda_fail(cudaGetLastError(), "launch");
}

// Host rays of a large query: they go to the device in chunks on the context's copy
// stream, and each chunk is traced as soon as it has landed while the next is still on
// the way; host results go back chunk by chunk behind their traces.  Every copy back is
// issued after every copy in, so a pageable output (whose copy waits for the host) does
// not hold up the inputs.  Results are per ray, so they equal the one-launch query's.
constexpr int kPipeChunks = 4;
constexpr int32_t kPipeMinRays = 1 << 20;

bool use_pipeline(const lux_ctx* ctx, const float* rays, int32_t nrays) {
    return nrays >= kPipeMinRays && pointer_kind(rays, ctx->device) == PtrKind::kHost;
}

int ensure_pipeline(lux_ctx* ctx) {
    if (ctx->copy_stream) return LUX_OK;
    cudaError_t err = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
    for (cudaEvent_t& e : ctx->pipe_events)
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return lux::cuda_fail(err, "copy stream");
}

template <bool kAny>
int trace_pipelined(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int32_t nrays,
                    int32_t* hit_id, float* hit_t) {
    static_assert(2 * kPipeChunks + 2 <= 16, "pipeline events");
    if (int st = ensure_pipeline(ctx)) return st;
    const size_t r = static_cast<size_t>(nrays);
    Staging staging(ctx);  // device room only: the copies are issued here, chunk by chunk
    void *d_rays = nullptr, *d_id = nullptr, *d_t = nullptr;
    staging.add(rays, 32 * r, false, false, &d_rays);
    staging.add(hit_id, 4 * r, false, false, &d_id);
    if (!kAny) staging.add(hit_t, 4 * r, false, false, &d_t);
    int st = staging.begin();
    if (st) return st;
    const bool id_back = d_id != hit_id;
    const bool t_back = !kAny && hit_t && d_t != hit_t;
    cudaStream_t s = ctx->stream, c = ctx->copy_stream;
    cudaEvent_t* ev = ctx->pipe_events;  // 0 start, 1..K copied in, K+1..2K traced, 2K+1 end
    const int32_t chunk = (nrays + kPipeChunks - 1) / kPipeChunks;
    // The copy stream starts after the work already queued on the context's stream.
    cudaError_t err = cudaEventRecord(ev[0], s);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(c, ev[0], 0);
    for (int k = 0; k < kPipeChunks && err == cudaSuccess; ++k) {
        const int32_t lo = k * chunk, cnt = std::min(chunk, nrays - lo);
        if (cnt <= 0) break;
        err = cudaMemcpyAsync(static_cast<char*>(d_rays) + 32 * size_t(lo),
                              reinterpret_cast<const char*>(rays) + 32 * size_t(lo),
                              32 * size_t(cnt), cudaMemcpyHostToDevice, c);
        if (err == cudaSuccess) err = cudaEventRecord(ev[1 + k], c);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(s, ev[1 + k], 0);
        if (err != cudaSuccess) break;
        const float* kr = static_cast<const float*>(d_rays) + 8 * size_t(lo);
        int* kid = static_cast<int*>(d_id) + lo;
        st = kAny ? lux::trace_any(ctx, bvh, kr, cnt, kid)
                  : lux::trace_closest(ctx, bvh, kr, cnt, kid,
                                       d_t ? static_cast<float*>(d_t) + lo : nullptr);
        if (st) {
            cudaStreamSynchronize(c);  // no copy may still read the caller's rays
            return st;
        }
        err = cudaEventRecord(ev[1 + kPipeChunks + k], s);
    }
    for (int k = 0; k < kPipeChunks && err == cudaSuccess && (id_back || t_back); ++k) {
        const int32_t lo = k * chunk, cnt = std::min(chunk, nrays - lo);
        if (cnt <= 0) break;
        err = cudaStreamWaitEvent(c, ev[1 + kPipeChunks + k], 0);
        if (err == cudaSuccess && id_back)
            err = cudaMemcpyAsync(hit_id + lo, static_cast<int*>(d_id) + lo, 4 * size_t(cnt),
                                  cudaMemcpyDeviceToHost, c);
        if (err == cudaSuccess && t_back)
            err = cudaMemcpyAsync(hit_t + lo, static_cast<float*>(d_t) + lo, 4 * size_t(cnt),
                                  cudaMemcpyDeviceToHost, c);
    }
    // Later work on the context's stream (and the wait below) comes after the copies.
    if (err == cudaSuccess) err = cudaEventRecord(ev[2 * kPipeChunks + 1], c);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(s, ev[2 * kPipeChunks + 1], 0);
    if (err != cudaSuccess) {
        cudaStreamSynchronize(c);
        return lux::cuda_fail(err, "chunked ray query");
    }
    return sync_and_check(ctx);
}

}  // namespace

namespace lux {

int fail(int status, const std::string& message) {
    g_error = message;
    return status;
}

int cuda_fail(cudaError_t err, const char* what) {
    if (err == cudaSuccess) return LUX_OK;
    g_error = std::string(what) + ": " + cudaGetErrorString(err);
    return err == cudaErrorMemoryAllocation ? LUX_ERR_OUT_OF_MEMORY : LUX_ERR_CUDA;
}

int ensure_scratch(lux_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->scratch_bytes) return LUX_OK;
    if (ctx->scratch) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->scratch);
        ctx->scratch = nullptr;
        ctx->scratch_bytes = 0;
    }
    size_t want = std::max(bytes, size_t(1) << 20);
    cudaError_t err = cudaMalloc(&ctx->scratch, want);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return fail(LUX_ERR_OUT_OF_MEMORY, "scratch allocation failed");
    }
    ctx->scratch_bytes = want;
    return LUX_OK;
}

}  // namespace lux

extern "C" {

int lux_abi_version(void) { return LUX_ABI_VERSION; }

const char* lux_last_error(void) { return g_error.c_str(); }

int lux_ctx_create(lux_ctx** out, int device, void* stream) {
    if (!out) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null output");
    *out = nullptr;
    int count = 0;
    cudaError_t err = cudaGetDeviceCount(&count);
    if (err != cudaSuccess) return lux::cuda_fail(err, "cudaGetDeviceCount");
    if (device < 0 || device >= count)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "device index out of range");
    err = cudaSetDevice(device);
    if (err != cudaSuccess) return lux::cuda_fail(err, "cudaSetDevice");
    lux_ctx* ctx = new (std::nothrow) lux_ctx();
    if (!ctx) return lux::fail(LUX_ERR_OUT_OF_MEMORY, "context allocation failed");
    ctx->device = device;
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (stream) {
        ctx->stream = static_cast<cudaStream_t>(stream);
    } else {
        err = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
        if (err != cudaSuccess) {
            delete ctx;
            return lux::cuda_fail(err, "cudaStreamCreate");
        }
        ctx->stream = ctx->own_stream;
    }
    err = cudaMalloc(&ctx->d_error, sizeof(int));
    if (err == cudaSuccess) err = cudaMemset(ctx->d_error, 0, sizeof(int));
    if (err == cudaSuccess) err = cudaMalloc(&ctx->d_counter, 64);
    if (err == cudaSuccess) err = cudaMemset(ctx->d_counter, 0, 64);
    if (err != cudaSuccess) {
        if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
        delete ctx;
        return lux::cuda_fail(err, "context init");
    }
    *out = ctx;
    return LUX_OK;
}

int lux_ctx_destroy(lux_ctx* ctx) {
    if (!ctx) return LUX_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->staging) cudaFree(ctx->staging);
    if (ctx->d_error) cudaFree(ctx->d_error);
    if (ctx->d_counter) cudaFree(ctx->d_counter);
    lux::render_runtime_free(ctx);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
        for (cudaEvent_t e : ctx->pipe_events)
            if (e) cudaEventDestroy(e);
    }
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return LUX_OK;
}

int lux_ctx_set_option(lux_ctx* ctx, int32_t option, int64_t value) {
    if (!ctx) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null context");
    switch (option) {
        case LUX_OPT_TRACE_VARIANT:
            if (value < 0 || value > 4) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "trace variant 0..4");
            ctx->trace_variant = static_cast<int>(value);
            return LUX_OK;
        case LUX_OPT_TRACE_BUDGET:
            if (value < 1 || value > 4096) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "trace budget 1..4096");
            ctx->trace_budget = static_cast<int>(value);
            return LUX_OK;
        case LUX_OPT_PATH_BUDGET:
            if (value < 1 || value > 4096) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "path budget 1..4096");
            ctx->path_budget = static_cast<int>(value);
            return LUX_OK;
        case LUX_OPT_RENDER_BATCH:
            if (value < 1 || value > (1 << 28)) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "render batch 1..2^28");
            ctx->render_batch = static_cast<int>(value);
            return LUX_OK;
        case LUX_OPT_REFILL_BLOCKS:
            if (value < 0 || value > 3) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "refill blocks 0..3");
            ctx->refill_blocks = static_cast<int>(value);
            return LUX_OK;
        default:
            return lux::fail(LUX_ERR_INVALID_ARGUMENT, "unknown option");
    }
}

int lux_ctx_get_option(lux_ctx* ctx, int32_t option, int64_t* value) {
    if (!ctx || !value) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    switch (option) {
        case LUX_OPT_TRACE_VARIANT: *value = ctx->trace_variant; return LUX_OK;
        case LUX_OPT_TRACE_BUDGET: *value = ctx->trace_budget; return LUX_OK;
        case LUX_OPT_RENDER_BATCH: *value = ctx->render_batch; return LUX_OK;
        case LUX_OPT_PATH_BUDGET: *value = ctx->path_budget; return LUX_OK;
        case LUX_OPT_REFILL_BLOCKS: *value = ctx->refill_blocks; return LUX_OK;
        case LUX_OPT_SCRATCH_BYTES: *value = static_cast<int64_t>(ctx->scratch_bytes); return LUX_OK;
        case LUX_OPT_STAGING_BYTES: *value = static_cast<int64_t>(ctx->staging_bytes); return LUX_OK;
        default: return lux::fail(LUX_ERR_INVALID_ARGUMENT, "unknown option");
    }
}

int lux_ctx_set_stream(lux_ctx* ctx, void* stream) {
    if (int st = check_ctx(ctx)) return st;
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    if (!ctx->stream) {
        cudaError_t err = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
        if (err != cudaSuccess) return lux::cuda_fail(err, "cudaStreamCreate");
        ctx->stream = ctx->own_stream;
    }
    return LUX_OK;
}

int lux_ctx_synchronize(lux_ctx* ctx) {
    if (int st = check_ctx(ctx)) return st;
    return sync_and_check(ctx);
}

int lux_ctx_launch_count(lux_ctx* ctx, int64_t* count) {
    if (!ctx || !count) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    *count = ctx->launches;
    return LUX_OK;
}

int lux_lbvh_build(lux_ctx* ctx, const float* prims, int32_t n, int32_t kind,
                   int32_t morton_bits, lux_bvh** out) {
    if (int st = check_ctx(ctx)) return st;
    if (!out) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null output");
    *out = nullptr;
    if (n < 0 || (n > 0 && !prims)) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "bad primitive array");
    if (n > (1 << 30)) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "too many primitives (max 2^30)");
    if (kind != LUX_PRIM_TRIANGLES && kind != LUX_PRIM_AABBS)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "unknown primitive kind");
    if (morton_bits != 30 && morton_bits != 63)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "morton_bits must be 30 or 63");
    lux_bvh* bvh = new (std::nothrow) lux_bvh();
    if (!bvh) return lux::fail(LUX_ERR_OUT_OF_MEMORY, "bvh allocation failed");
    bvh->n = n;
    bvh->kind = kind;
    bvh->morton_bits = morton_bits;
    bvh->device = ctx->device;
    bvh->has_triangles = kind == LUX_PRIM_TRIANGLES;
    int st = lux::lbvh_alloc(ctx, bvh);
    if (st) {
        delete bvh;
        return st;
    }
    size_t per = kind == LUX_PRIM_TRIANGLES ? 9 : 6;
    Staging staging(ctx);
    void* d_prims = nullptr;
    staging.add(prims, sizeof(float) * per * static_cast<size_t>(n), true, false, &d_prims);
    st = staging.begin();
    if (!st) st = lux::lbvh_build(ctx, bvh, static_cast<const float*>(d_prims));
    if (!st) st = finish_call(ctx, staging);
    // Host-staged inputs must outlive the kernels that read them.
    if (!st && !staging.items.empty()) st = sync_and_check(ctx);
    if (st) {
        lux::lbvh_free(bvh);
        delete bvh;
        return st;
    }
    *out = bvh;
    return LUX_OK;
}

int lux_lbvh_rebuild(lux_ctx* ctx, lux_bvh* bvh, const float* prims, int32_t n) {
    if (int st = check_ctx(ctx)) return st;
    if (!bvh) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null bvh");
    if (n < 0 || (n > 0 && !prims)) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "bad primitive array");
    if (n > (1 << 30)) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "too many primitives (max 2^30)");
    if (n > bvh->capacity) {
        cudaStreamSynchronize(ctx->stream);
        lux::lbvh_free(bvh);
        bvh->capacity = 0;
        bvh->n = n;
        if (int st = lux::lbvh_alloc(ctx, bvh)) {
            bvh->n = 0;
            return st;
        }
    }
    bvh->n = n;
    bvh->has_triangles = bvh->kind == LUX_PRIM_TRIANGLES;  // attached triangles go stale
    size_t per = bvh->kind == LUX_PRIM_TRIANGLES ? 9 : 6;
    Staging staging(ctx);
    void* d_prims = nullptr;
    staging.add(prims, sizeof(float) * per * static_cast<size_t>(n), true, false, &d_prims);
    int st = staging.begin();
    if (!st) st = lux::lbvh_build(ctx, bvh, static_cast<const float*>(d_prims));
    if (!st) st = finish_call(ctx, staging);
    if (!st && !staging.items.empty()) st = sync_and_check(ctx);
    return st;
}

int lux_lbvh_refit(lux_ctx* ctx, lux_bvh* bvh, const float* prims, int32_t n) {
    if (int st = check_ctx(ctx)) return st;
    if (!bvh) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null bvh");
    if (n != bvh->n) return lux::fail(LUX_ERR_MISMATCH, "refit primitive count differs from build");
    if (n > 0 && !prims) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "bad primitive array");
    size_t per = bvh->kind == LUX_PRIM_TRIANGLES ? 9 : 6;
    Staging staging(ctx);
    void* d_prims = nullptr;
    staging.add(prims, sizeof(float) * per * static_cast<size_t>(n), true, false, &d_prims);
    int st = staging.begin();
    if (!st) st = lux::lbvh_refit(ctx, bvh, static_cast<const float*>(d_prims));
    if (!st) st = finish_call(ctx, staging);
    if (!st && !staging.items.empty()) st = sync_and_check(ctx);
    return st;
}

int lux_bvh_attach_triangles(lux_ctx* ctx, lux_bvh* bvh, const float* tris, int32_t n) {
    if (int st = check_ctx(ctx)) return st;
    if (!bvh) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null bvh");
    if (n != bvh->n) return lux::fail(LUX_ERR_MISMATCH, "triangle count differs from the BVH's");
    if (n > 0 && !tris) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null triangles");
    Staging staging(ctx);
    void* d_tris = nullptr;
    staging.add(tris, sizeof(float) * 9 * static_cast<size_t>(n), true, false, &d_tris);
    int st = staging.begin();
    if (!st) st = lux::lbvh_attach_triangles(ctx, bvh, static_cast<const float*>(d_tris));
    if (!st) st = finish_call(ctx, staging);
    if (!st && !staging.items.empty()) st = sync_and_check(ctx);
    if (!st) bvh->has_triangles = true;
    return st;
}

int lux_bvh_destroy(lux_bvh* bvh) {
    if (!bvh) return LUX_OK;
    cudaSetDevice(bvh->device);
    lux::lbvh_free(bvh);
    delete bvh;
    return LUX_OK;
}

int lux_bvh_info(lux_ctx* ctx, const lux_bvh* bvh, int32_t* n, int32_t* kind,
                 int32_t* morton_bits, float* root_bounds) {
    if (int st = check_ctx(ctx)) return st;
    if (!bvh) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null bvh");
    if (n) *n = bvh->n;
    if (kind) *kind = bvh->kind;
    if (morton_bits) *morton_bits = bvh->morton_bits;
    if (root_bounds) {
        if (bvh->n <= 0) {
            for (int a = 0; a < 3; ++a) {
                root_bounds[a] = INFINITY;
                root_bounds[3 + a] = -INFINITY;
            }
            return LUX_OK;
        }
        Staging staging(ctx);
        void* d_root = nullptr;
        staging.add(root_bounds, sizeof(float) * 6, false, true, &d_root);
        int st = staging.begin();
        if (st) return st;
        cudaError_t err = cudaMemcpyAsync(d_root, bvh->root, sizeof(float) * 6,
                                          cudaMemcpyDeviceToDevice, ctx->stream);
        if (err != cudaSuccess) return lux::cuda_fail(err, "root copy");
        return finish_call(ctx, staging);
    }
    return LUX_OK;
}

// Allocation-free Morton sort: argument checks here, the work and the static array's
// per-device set-up in lbvh.cu.
int lux_lbvh_morton_sort_static(lux_ctx* ctx, const float* prims, int32_t n, int32_t kind,
                                int32_t morton_bits, uint64_t* sorted_codes,
                                int32_t* sorted_ids) {
    if (int st = check_ctx(ctx)) return st;
    if (kind != LUX_PRIM_TRIANGLES && kind != LUX_PRIM_AABBS)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "unknown primitive kind");
    if (morton_bits != 30 && morton_bits != 63)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "morton_bits must be 30 or 63");
    if (n > LUX_STATIC_SORT_MAX_PRIMS)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT,
                         "lux_lbvh_morton_sort_static: " + std::to_string(n) +
                             " primitives exceed LUX_STATIC_SORT_MAX_PRIMS (" +
                             std::to_string(LUX_STATIC_SORT_MAX_PRIMS) + ")");
    if (n < 0) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "negative primitive count");
    if (n > 0 && (!is_device_pointer(prims, ctx->device) ||
                  !is_device_pointer(sorted_codes, ctx->device) ||
                  !is_device_pointer(sorted_ids, ctx->device)))
        return lux::fail(LUX_ERR_INVALID_ARGUMENT,
                         "lux_lbvh_morton_sort_static takes device pointers on the context's "
                         "device only");
    return lux::lbvh_morton_sort_static(ctx, prims, n, kind, morton_bits, sorted_codes,
                                        sorted_ids);
}

int lux_bvh_download(lux_ctx* ctx, const lux_bvh* bvh, uint64_t* sorted_codes,
                     int32_t* sorted_ids, int32_t* node_left, int32_t* node_right,
                     float* node_bounds) {
    if (int st = check_ctx(ctx)) return st;
    if (!bvh) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null bvh");
    size_t n = static_cast<size_t>(bvh->n);
    if (n == 0) return LUX_OK;
    size_t count = 2 * n - 1;
    Staging staging(ctx);
    void *d_codes, *d_ids, *d_left, *d_right, *d_bounds;
    staging.add(sorted_codes, 8 * n, false, true, &d_codes);
    staging.add(sorted_ids, 4 * n, false, true, &d_ids);
    staging.add(node_left, 4 * count, false, true, &d_left);
    staging.add(node_right, 4 * count, false, true, &d_right);
    staging.add(node_bounds, 24 * count, false, true, &d_bounds);
    int st = staging.begin();
    if (st) return st;
    if (d_ids) {
        cudaError_t err = cudaMemcpyAsync(d_ids, bvh->sorted_ids, 4 * n,
                                          cudaMemcpyDeviceToDevice, ctx->stream);
        if (err != cudaSuccess) return lux::cuda_fail(err, "sorted id copy");
    }
    st = lux::lbvh_export(ctx, bvh, static_cast<uint64_t*>(d_codes), static_cast<int*>(d_left),
                          static_cast<int*>(d_right), static_cast<float*>(d_bounds));
    if (st) return st;
    return finish_call(ctx, staging);
}

static int check_query(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int32_t nrays) {
    if (int st = check_ctx(ctx)) return st;
    if (!bvh) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null bvh");
    if (!bvh->has_triangles)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT,
                         "ray queries need a triangle BVH (or lux_bvh_attach_triangles)");
    if (nrays < 0 || (nrays > 0 && !rays)) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "bad ray array");
    return LUX_OK;
}

int lux_trace_closest(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int32_t nrays,
                      int32_t* hit_id, float* hit_t) {
    if (int st = check_query(ctx, bvh, rays, nrays)) return st;
    if (nrays > 0 && !hit_id) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null hit_id");
    if (use_pipeline(ctx, rays, nrays)) return trace_pipelined<false>(ctx, bvh, rays, nrays, hit_id, hit_t);
    Staging staging(ctx);
    void *d_rays, *d_id, *d_t;
    size_t r = static_cast<size_t>(nrays);
    staging.add(rays, 32 * r, true, false, &d_rays);
    staging.add(hit_id, 4 * r, false, true, &d_id);
    staging.add(hit_t, 4 * r, false, true, &d_t);
    int st = staging.begin();
    if (st) return st;
    st = lux::trace_closest(ctx, bvh, static_cast<const float*>(d_rays), nrays,
                            static_cast<int*>(d_id), static_cast<float*>(d_t));
    if (st) return st;
    st = finish_call(ctx, staging);
    if (!st && !staging.items.empty() && !staging.has_host_output()) st = sync_and_check(ctx);
    return st;
}

int lux_trace_closest_stats(lux_ctx* ctx, const lux_bvh* bvh, const float* rays,
                            int32_t nrays, int64_t* totals) {
    if (int st = check_query(ctx, bvh, rays, nrays)) return st;
    if (!totals) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null totals");
    Staging staging(ctx);
    void *d_rays, *d_tot;
    staging.add(rays, 32 * static_cast<size_t>(nrays), true, false, &d_rays);
    staging.add(totals, 16, true, true, &d_tot);
    int st = staging.begin();
    if (st) return st;
    st = lux::trace_stats(ctx, bvh, static_cast<const float*>(d_rays), nrays,
                          static_cast<unsigned long long*>(d_tot));
    if (st) return st;
    return finish_call(ctx, staging);
}

int lux_trace_any(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int32_t nrays,
                  int32_t* hit_id) {
    if (int st = check_query(ctx, bvh, rays, nrays)) return st;
    if (nrays > 0 && !hit_id) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null hit_id");
    if (use_pipeline(ctx, rays, nrays)) return trace_pipelined<true>(ctx, bvh, rays, nrays, hit_id, nullptr);
    Staging staging(ctx);
    void *d_rays, *d_id;
    size_t r = static_cast<size_t>(nrays);
    staging.add(rays, 32 * r, true, false, &d_rays);
    staging.add(hit_id, 4 * r, false, true, &d_id);
    int st = staging.begin();
    if (st) return st;
    st = lux::trace_any(ctx, bvh, static_cast<const float*>(d_rays), nrays,
                        static_cast<int*>(d_id));
    if (st) return st;
    st = finish_call(ctx, staging);
    if (!st && !staging.items.empty() && !staging.has_host_output()) st = sync_and_check(ctx);
    return st;
}

static int overlap_common(lux_ctx* ctx, const lux_bvh* tree, const lux_bvh* queries, bool self,
                          int32_t* pairs, int64_t max_pairs, int64_t* found) {
    if (int st = check_ctx(ctx)) return st;
    if (!tree || !queries) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null bvh");
    if (max_pairs < 0 || (max_pairs > 0 && !pairs) || !found)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "bad pair buffer");
    Staging staging(ctx);
    void *d_pairs, *d_found;
    staging.add(pairs, 8 * static_cast<size_t>(max_pairs), false, true, &d_pairs);
    staging.add(found, 8, false, true, &d_found);
    int st = staging.begin();
    if (st) return st;
    st = lux::overlap(ctx, tree, queries, self, static_cast<int*>(d_pairs), max_pairs,
                      static_cast<unsigned long long*>(d_found));
    if (st) return st;
    return finish_call(ctx, staging);
}

int lux_overlap_self(lux_ctx* ctx, const lux_bvh* bvh, int32_t* pairs, int64_t max_pairs,
                     int64_t* found) {
    return overlap_common(ctx, bvh, bvh, true, pairs, max_pairs, found);
}

int lux_overlap_cross(lux_ctx* ctx, const lux_bvh* left, const lux_bvh* right,
                      int32_t* pairs, int64_t max_pairs, int64_t* found) {
    return overlap_common(ctx, left, right, false, pairs, max_pairs, found);
}

// ------------------------------------------------------------------ scenes and rendering

int lux_scene_create(lux_ctx* ctx, const lux_scene_desc* desc, lux_scene** out) {
    if (int st = check_ctx(ctx)) return st;
    if (!desc || !out) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    return lux::scene_create(ctx, desc, out);
}

int lux_camera_perspective(const float origin[3], const float look_at[3], float vfov_degrees,
                           float aspect, float lens_radius, float focal_distance,
                           lux_camera_desc* out) {
    if (!origin || !look_at || !out) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    return lux::camera_perspective(origin, look_at, vfov_degrees, aspect, lens_radius,
                                   focal_distance, out);
}

int lux_scene_destroy(lux_scene* scene) {
    if (!scene) return LUX_OK;
    cudaSetDevice(scene->device);
    cudaDeviceSynchronize();
    lux::scene_free(scene);
    delete scene;
    return LUX_OK;
}

int lux_scene_info(const lux_scene* scene, int32_t* triangles, int32_t* area_lights,
                   int32_t* lights) {
    if (!scene) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null scene");
    if (triangles) *triangles = scene->triangle_count;
    if (area_lights) *area_lights = scene->area_light_count;
    if (lights) *lights = scene->view.light_count;
    return LUX_OK;
}

int lux_scene_update_mesh(lux_ctx* ctx, lux_scene* scene, int32_t mesh, const float* vertices) {
    if (int st = check_ctx(ctx)) return st;
    if (!scene || !vertices) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    return lux::scene_update_mesh(ctx, scene, mesh, vertices);
}

static int render_common(lux_ctx* ctx, const lux_scene* scene, const lux_render_request* req,
                         float* out, bool per_sample) {
    if (int st = check_ctx(ctx)) return st;
    if (!scene || !req || !out) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    if (req->width <= 0 || req->height <= 0 || req->spp <= 0)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "render requires a non-empty film");
    if (req->max_depth < 0 || req->max_depth > 1000)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "max_depth must be in 0..1000");
    if (req->light_sampler < 0 || req->light_sampler > 2)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "light sampler: 0 uniform, 1 power or 2 tree");
    if (static_cast<long long>(req->width) * req->height > (1ll << 30))
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "image too large");
    size_t pixels = static_cast<size_t>(req->width) * req->height;
    size_t count = per_sample ? pixels * static_cast<size_t>(req->spp) : pixels;
    Staging staging(ctx);
    void* d_out = nullptr;
    staging.add(out, sizeof(float) * 3 * count, false, true, &d_out);
    int st = staging.begin();
    if (st) return st;
    st = lux::render(ctx, scene, *req, static_cast<float*>(d_out), per_sample);
    if (st) return st;
    st = finish_call(ctx, staging);
    if (st) return st;
    return sync_and_check(ctx);
}

int lux_render(lux_ctx* ctx, const lux_scene* scene, const lux_render_request* req,
               float* film_sum) {
    return render_common(ctx, scene, req, film_sum, false);
}

int lux_render_aovs(lux_ctx* ctx, const lux_scene* scene, const lux_render_request* req,
                    float* film_sum, float* shadow, float* ng, float* ns) {
    if (int st = check_ctx(ctx)) return st;
    if (!scene || !req || !film_sum) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    if (req->width <= 0 || req->height <= 0 || req->spp <= 0)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "render requires a non-empty film");
    if (req->max_depth < 0 || req->max_depth > 1000)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "max_depth must be in 0..1000");
    if (req->light_sampler < 0 || req->light_sampler > 2)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "light sampler: 0 uniform, 1 power or 2 tree");
    if (static_cast<long long>(req->width) * req->height > (1ll << 30))
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "image too large");
    const size_t bytes = sizeof(float) * 3 * static_cast<size_t>(req->width) * req->height;
    Staging staging(ctx);
    void *d_film = nullptr, *d_shadow = nullptr, *d_ng = nullptr, *d_ns = nullptr;
    staging.add(film_sum, bytes, false, true, &d_film);
    staging.add(shadow, bytes, false, true, &d_shadow);
    staging.add(ng, bytes, false, true, &d_ng);
    staging.add(ns, bytes, false, true, &d_ns);
    int st = staging.begin();
    if (st) return st;
    st = lux::render(ctx, scene, *req, static_cast<float*>(d_film), false,
                     static_cast<float*>(d_shadow), static_cast<float*>(d_ng),
                     static_cast<float*>(d_ns));
    if (st) return st;
    st = finish_call(ctx, staging);
    if (st) return st;
    return sync_and_check(ctx);
}

static_assert(sizeof(lux_path_log_record) == 152, "lux_path_log_record layout");

int lux_render_path_log(lux_ctx* ctx, const lux_scene* scene, const lux_render_request* req,
                        float* film_sum, lux_path_log_record* records, int64_t capacity,
                        int64_t* count) {
    if (int st = check_ctx(ctx)) return st;
    if (!scene || !req || !film_sum || !count || capacity < 0 || (capacity > 0 && !records))
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    if (req->width <= 0 || req->height <= 0 || req->spp <= 0)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "render requires a non-empty film");
    if (req->max_depth < 0 || req->max_depth > 1000)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "max_depth must be in 0..1000");
    if (req->light_sampler < 0 || req->light_sampler > 2)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "light sampler: 0 uniform, 1 power or 2 tree");
    if (static_cast<long long>(req->width) * req->height > (1ll << 30))
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "image too large");
    if (records && pointer_kind(records, ctx->device) != PtrKind::kHost)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "path log records must be host memory");
    const size_t bytes = sizeof(float) * 3 * static_cast<size_t>(req->width) * req->height;
    unsigned long long vertices = 0;
    Staging staging(ctx);
    void *d_film = nullptr, *d_records = nullptr, *d_count = nullptr;
    staging.add(film_sum, bytes, false, true, &d_film);
    staging.add(records, sizeof(lux_path_log_record) * static_cast<size_t>(capacity), false, true,
                &d_records);
    staging.add(&vertices, sizeof(vertices), false, true, &d_count);
    int st = staging.begin();
    if (st) return st;
    st = lux::render(ctx, scene, *req, static_cast<float*>(d_film), false, nullptr, nullptr,
                     nullptr, capacity > 0 ? static_cast<lux_path_log_record*>(d_records) : nullptr,
                     static_cast<unsigned long long*>(d_count), capacity);
    if (st) return st;
    st = finish_call(ctx, staging);
    if (st) return st;
    st = sync_and_check(ctx);
    if (st) return st;
    *count = static_cast<int64_t>(vertices);
    if (*count > capacity)
        return lux::fail(LUX_ERR_QUEUE_OVERFLOW, "path log capacity exhausted");
    // One path's vertices carry distinct ordinals, so the key is unique.
    std::sort(records, records + *count,
              [](const lux_path_log_record& a, const lux_path_log_record& b) {
                  if (a.sample_index != b.sample_index) return a.sample_index < b.sample_index;
                  if (a.pixel_index != b.pixel_index) return a.pixel_index < b.pixel_index;
                  return a.vertex < b.vertex;
              });
    return LUX_OK;
}

int lux_render_samples(lux_ctx* ctx, const lux_scene* scene, const lux_render_request* req,
                       float* samples) {
    return render_common(ctx, scene, req, samples, true);
}

int lux_scene_select_lights(lux_ctx* ctx, const lux_scene* scene, int32_t light_sampler,
                            const float* positions, const float* select_u, int32_t n,
                            int32_t* light_index, float* pmf, float* eval_pmf) {
    if (int st = check_ctx(ctx)) return st;
    if (!scene || n < 0 || (n > 0 && (!positions || !select_u || !light_index || !pmf || !eval_pmf)))
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    if (light_sampler < 0 || light_sampler > 2)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "light sampler: 0 uniform, 1 power or 2 tree");
    if (n == 0) return LUX_OK;
    const size_t count = static_cast<size_t>(n);
    Staging staging(ctx);
    void *d_pos = nullptr, *d_u = nullptr, *d_index = nullptr, *d_pmf = nullptr, *d_eval = nullptr;
    staging.add(positions, sizeof(float) * 3 * count, true, false, &d_pos);
    staging.add(select_u, sizeof(float) * count, true, false, &d_u);
    staging.add(light_index, sizeof(int32_t) * count, false, true, &d_index);
    staging.add(pmf, sizeof(float) * count, false, true, &d_pmf);
    staging.add(eval_pmf, sizeof(float) * count, false, true, &d_eval);
    int st = staging.begin();
    if (st) return st;
    st = lux::select_lights(ctx, scene, light_sampler, static_cast<const float*>(d_pos),
                            static_cast<const float*>(d_u), n, static_cast<int32_t*>(d_index),
                            static_cast<float*>(d_pmf), static_cast<float*>(d_eval));
    if (st) return st;
    st = finish_call(ctx, staging);
    if (st) return st;
    return sync_and_check(ctx);
}

int lux_render_traversal_stats(lux_ctx* ctx, const lux_scene* scene,
                               const lux_render_request* req, float* film_sum,
                               int64_t* stats) {
    if (int st = check_ctx(ctx)) return st;
    if (!scene || !req || !film_sum || !stats)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    if (req->width <= 0 || req->height <= 0 || req->spp <= 0)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "render requires a non-empty film");
    if (req->max_depth < 0 || req->max_depth > 1000)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "max_depth must be in 0..1000");
    if (req->light_sampler < 0 || req->light_sampler > 2)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "light sampler: 0 uniform, 1 power or 2 tree");
    if (static_cast<long long>(req->width) * req->height > (1ll << 30))
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "image too large");
    const size_t bytes = sizeof(float) * 3 * static_cast<size_t>(req->width) * req->height;
    unsigned long long walk[3] = {0, 0, 0};
    Staging staging(ctx);
    void *d_film = nullptr, *d_walk = nullptr;
    staging.add(film_sum, bytes, false, true, &d_film);
    staging.add(walk, sizeof(walk), false, true, &d_walk);
    int st = staging.begin();
    if (st) return st;
    st = lux::render(ctx, scene, *req, static_cast<float*>(d_film), false, nullptr, nullptr,
                     nullptr, nullptr, nullptr, 0, static_cast<unsigned long long*>(d_walk));
    if (st) return st;
    st = finish_call(ctx, staging);
    if (st) return st;
    st = sync_and_check(ctx);
    if (st) return st;
    int64_t rays[2];
    lux::render_ray_counts(ctx, rays);
    stats[0] = rays[0];
    stats[1] = rays[1];
    for (int k = 0; k < 3; ++k) stats[2 + k] = static_cast<int64_t>(walk[k]);
    return LUX_OK;
}

int lux_render_ray_counts(lux_ctx* ctx, int64_t* counts) {
    if (!ctx || !counts) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    return lux::render_ray_counts(ctx, counts);
}

}  // extern "C"
