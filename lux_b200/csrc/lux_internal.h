// Host-side internals shared by the C-ABI layer and the kernel launchers.
#pragma once

#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "lux_bvh.cuh"

struct lux_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int sm_count = 148;
    int* d_error = nullptr;          // device error word (lux::kErr* bits)
    int64_t launches = 0;            // kernels launched through this context
    unsigned* d_counter = nullptr;   // device work counter (persistent kernels)
    // Tunables (lux_ctx_set_option).
    int trace_variant = 0;           // lux::kTrace* (auto: wide persistent)
    int trace_budget = 16;           // traversal steps per refill round (ray queries)
    int path_budget = 32;            // traversal steps per refill round (path tracer)
    int render_batch = 1 << 22;      // paths in flight per wavefront batch
    int refill_blocks = 0;           // blocks per SM of the refilling kernels (0: max)
    void* render_runtime = nullptr;  // wavefront buffers, grown on demand
    // Growable device scratch, reused across calls on this context.
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    // Growable device staging for host inputs / outputs.
    void* staging = nullptr;
    size_t staging_bytes = 0;
    // Copy stream and events of the chunked host-ray queries (created on first use).
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t pipe_events[16] = {};
    // Resident blocks per SM of the persistent kernels on this context's device, by
    // lux::kOcc* slot, measured on first launch (0: not yet).  Per context, so per device
    // and under the one-thread-per-context rule of the ABI.
    int occupancy[8] = {};
};

struct lux_bvh {
    int n = 0;
    int capacity = 0;       // primitives the device storage can hold
    bool has_triangles = false;  // TriRecord array valid (triangle BVHs, or attached)
    int kind = 0;           // LUX_PRIM_TRIANGLES / LUX_PRIM_AABBS
    int morton_bits = 30;
    int device = 0;
    lux::BvhNode* nodes = nullptr;      // n - 1
    lux::TriRecord* tris = nullptr;     // n (triangle BVHs)
    int* sorted_ids = nullptr;          // n
    int* leaf_parent = nullptr;         // n
    int* node_parent = nullptr;         // n - 1
    int4* node_info = nullptr;          // n - 1: first and last sorted leaf, parent code
    unsigned* flags = nullptr;          // n - 1, zero between passes
    void* codes = nullptr;              // n sorted codes (uint32 or uint64)
    float* root = nullptr;              // 6
    lux::WideNode* wide = nullptr;      // capacity - 1, built on demand for ray queries
    bool wide_current = false;          // wide matches nodes (cleared by build/refit)
    int wide_capacity = 0;              // wide nodes allocated
    lux::BvhView view() const {
        lux::BvhView v;
        v.nodes = nodes;
        v.wide = wide;
        v.tris = tris;
        v.sorted_ids = sorted_ids;
        v.leaf_parent = leaf_parent;
        v.root = root;
        v.n = n;
        v.leaf_is_triangle_box = kind == LUX_PRIM_TRIANGLES;
        return v;
    }
};

namespace lux {

enum : int {
    kTraceAuto = 0,
    kTraceStatic = 1,
    kTracePersistent = 2,
    kTraceWide = 3,
    kTraceWidePersistent = 4
};

// Slots of lux_ctx::occupancy.
enum : int {
    kOccWideClosest = 0,
    kOccWideAny = 1,
    kOccPersistClosest = 2,
    kOccPersistAny = 3,
    kOccExtendRefill = 4,
    kOccShadowRefill = 5
};

// Resident blocks per SM of `kernel` at `threads` threads on the context's device (at
// least 1), measured once per context.
template <typename Kernel>
inline int occupancy_blocks(lux_ctx* ctx, int slot, Kernel kernel, int threads) {
    int& v = ctx->occupancy[slot];
    if (v == 0) {
        int blocks = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, 0) !=
            cudaSuccess) {
            cudaGetLastError();
            blocks = 0;
        }
        v = blocks > 0 ? blocks : 1;
    }
    return v;
}

// Status helpers (defined in capi.cu).
int fail(int status, const std::string& message);
int cuda_fail(cudaError_t err, const char* what);
int ensure_scratch(lux_ctx* ctx, size_t bytes);

// LBVH (lbvh.cu).  prims are device pointers.
int lbvh_alloc(lux_ctx* ctx, lux_bvh* bvh);
int lbvh_build(lux_ctx* ctx, lux_bvh* bvh, const float* prims);
int lbvh_refit(lux_ctx* ctx, lux_bvh* bvh, const float* prims);
// Brings the 4-wide nodes up to date with the binary nodes (stream-ordered; allocates
// them on first use).  Every ray query calls it; builds and refits mark them stale.
int lbvh_ensure_wide(lux_ctx* ctx, lux_bvh* bvh);
void lbvh_free(lux_bvh* bvh);
int lbvh_export(lux_ctx* ctx, const lux_bvh* bvh, uint64_t* codes64, int* left, int* right,
                float* bounds);
size_t lbvh_scratch_bytes(int n, int morton_bits);
// Morton codes and their stable sort into caller device arrays, temporaries in the
// module's static array (no device allocation; synchronous).
int lbvh_morton_sort_static(lux_ctx* ctx, const float* prims, int n, int kind, int morton_bits,
                            uint64_t* sorted_codes, int* sorted_ids);
int lbvh_attach_triangles(lux_ctx* ctx, lux_bvh* bvh, const float* tris);

// Queries (traverse.cu).  All pointers are device pointers.
int trace_closest(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int nrays, int* hit_id,
                  float* hit_t);
int trace_any(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int nrays, int* hit_id);
int trace_stats(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int nrays,
                unsigned long long* totals);
int overlap(lux_ctx* ctx, const lux_bvh* tree, const lux_bvh* queries, bool self, int* pairs,
            int64_t max_pairs, unsigned long long* d_found);

}  // namespace lux
