// BVH validators: lux_bvh_validate_structure and lux_bvh_validate_primitives.
//
// Host checks over the downloaded tree, restating validate_gpu_bvh_structure and
// validate_gpu_bvh_matches_primitives (bvh/gpu_bvh.cu:667-891) on this library's layout:
// Karras internal nodes 0..n-2 with both child boxes, leaves in sorted order, parent
// links coded (parent << 1) | slot.  The messages are the reference's, so a caller that
// prints them sees the same text.  The checks that only concern the reference's
// stackless preorder array (escape indices) have no counterpart here; their role, every
// node reached exactly once from the root, is covered by the parent/child and traversal
// checks.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lux_gpu.h"
#include "lux_internal.h"

namespace {

struct HostBox {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void expand(const HostBox& b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::fmin(lo[a], b.lo[a]);
            hi[a] = std::fmax(hi[a], b.hi[a]);
        }
    }
};

HostBox box_at(const float* six) {
    HostBox b;
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = six[a];
        b.hi[a] = six[3 + a];
    }
    return b;
}

// aabb_close (bvh/gpu_bvh.cu:392-395): squared corner distances within 1e-4^2.
bool aabb_close(const HostBox& a, const HostBox& b, float eps = 1e-4f) {
    float dl = 0, dh = 0;
    for (int k = 0; k < 3; ++k) {
        dl += (a.lo[k] - b.lo[k]) * (a.lo[k] - b.lo[k]);
        dh += (a.hi[k] - b.hi[k]) * (a.hi[k] - b.hi[k]);
    }
    return dl <= eps * eps && dh <= eps * eps;
}

struct Downloaded {
    int n = 0;
    std::vector<uint64_t> codes;
    std::vector<int32_t> ids, left, right, leaf_parent, node_parent;
    std::vector<float> bounds;  // (2n-1) x 6, host tree layout
    HostBox root;
};

int download(lux_ctx* ctx, const lux_bvh* bvh, Downloaded& d) {
    const int n = bvh->n;
    d.n = n;
    const size_t count = 2 * size_t(n) - 1;
    d.codes.resize(n);
    d.ids.resize(n);
    d.left.resize(count);
    d.right.resize(count);
    d.bounds.resize(6 * count);
    int st = lux_bvh_download(ctx, bvh, d.codes.data(), d.ids.data(), d.left.data(),
                              d.right.data(), d.bounds.data());
    if (st) return st;
    d.leaf_parent.resize(n);
    d.node_parent.resize(std::max(n - 1, 0));
    float root[6];
    cudaError_t err = cudaMemcpy(d.leaf_parent.data(), bvh->leaf_parent, sizeof(int) * n,
                                 cudaMemcpyDeviceToHost);
    if (err == cudaSuccess && n > 1)
        err = cudaMemcpy(d.node_parent.data(), bvh->node_parent, sizeof(int) * (n - 1),
                         cudaMemcpyDeviceToHost);
    if (err == cudaSuccess)
        err = cudaMemcpy(root, bvh->root, sizeof(root), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return lux::cuda_fail(err, "validator download");
    d.root = box_at(root);
    return LUX_OK;
}

// Child of internal node p in the host layout (internal i, or leaf k as n-1+k) at slot.
int child_of(const Downloaded& d, int p, int slot) { return slot ? d.right[p] : d.left[p]; }

// Returns the empty string when the structure is valid, else the reference's message.
std::string check_structure(const Downloaded& d) {
    const int n = d.n;
    const int internal_count = n - 1;
    std::vector<int> seen(n, 0);
    for (int i = 0; i < n; ++i) {
        int input = d.ids[i];
        if (input < 0 || input >= n) return "sorted input index out of range";
        if (++seen[input] != 1) return "duplicate sorted input index";
    }
    HostBox expected_root;
    for (int k = 0; k < n; ++k) expected_root.expand(box_at(&d.bounds[6 * (size_t(n) - 1 + k)]));
    if (!aabb_close(expected_root, d.root)) return "root bounds mismatch";
    if (!aabb_close(box_at(&d.bounds[0]), d.root)) return "stackless root bounds mismatch";
    if (n == 1) {
        if (d.ids[0] != 0 || d.leaf_parent[0] != -1) return "single leaf stackless node mismatch";
        return "";
    }
    for (int i = 1; i < n; ++i)
        if (d.codes[i - 1] > d.codes[i]) return "Morton codes are not sorted";
    int leaf_refs = 0;
    for (int p = 0; p < internal_count; ++p)
        for (int slot = 0; slot < 2; ++slot)
            if (child_of(d, p, slot) >= internal_count) ++leaf_refs;
    if (leaf_refs != n) return "stackless leaf count mismatch";
    for (int child = 1; child < internal_count; ++child) {
        int code = d.node_parent[child];
        int parent = code >> 1;
        if (code < 0 || parent >= internal_count) return "internal parent index out of range";
        if (child_of(d, parent, code & 1) != child) return "internal parent/child mismatch";
    }
    for (int leaf = 0; leaf < n; ++leaf) {
        int code = d.leaf_parent[leaf];
        int parent = code >> 1;
        if (code < 0 || parent >= internal_count) return "leaf parent index out of range";
        if (child_of(d, parent, code & 1) != internal_count + leaf) return "leaf parent/child mismatch";
    }
    std::vector<int> stack{0};
    std::vector<int> visited_internal(internal_count, 0), visited_leaf(n, 0);
    while (!stack.empty()) {
        int node = stack.back();
        stack.pop_back();
        if (node >= internal_count) {
            int leaf = node - internal_count;
            if (leaf < 0 || leaf >= n || ++visited_leaf[leaf] != 1)
                return "invalid or duplicate leaf traversal";
            continue;
        }
        if (node < 0 || ++visited_internal[node] != 1) return "invalid or duplicate internal traversal";
        stack.push_back(d.right[node]);
        stack.push_back(d.left[node]);
    }
    for (int i = 0; i < internal_count; ++i)
        if (visited_internal[i] != 1) return "unvisited internal node";
    for (int i = 0; i < n; ++i)
        if (visited_leaf[i] != 1) return "unvisited leaf node";
    return "";
}

void report(bool ok, const std::string& message, int32_t* valid, char* out, int32_t capacity) {
    *valid = ok ? 1 : 0;
    if (out && capacity > 0) {
        size_t len = std::min<size_t>(message.size(), size_t(capacity) - 1);
        std::memcpy(out, message.data(), len);
        out[len] = '\0';
    }
}

}  // namespace

extern "C" {

int lux_bvh_validate_structure(lux_ctx* ctx, const lux_bvh* bvh, int32_t* valid, char* message,
                               int32_t message_capacity) {
    if (!ctx || !valid) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    if (cudaError_t err = cudaSetDevice(ctx->device)) return lux::cuda_fail(err, "cudaSetDevice");
    if (!bvh || bvh->n <= 0) {
        report(false, "BVH is not valid", valid, message, message_capacity);
        return LUX_OK;
    }
    Downloaded d;
    if (int st = download(ctx, bvh, d)) return st;
    std::string why = check_structure(d);
    report(why.empty(), why, valid, message, message_capacity);
    return LUX_OK;
}

int lux_bvh_validate_primitives(lux_ctx* ctx, const lux_bvh* bvh, const float* prims, int32_t n,
                                int32_t* valid, char* message, int32_t message_capacity) {
    if (!ctx || !valid || n < 0 || (n > 0 && !prims))
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "bad argument");
    if (cudaError_t err = cudaSetDevice(ctx->device)) return lux::cuda_fail(err, "cudaSetDevice");
    if (n == 0) {
        bool ok = !bvh || bvh->n == 0;
        report(ok, ok ? "" : "BVH contains primitives for an empty scene", valid, message,
               message_capacity);
        return LUX_OK;
    }
    if (!bvh || bvh->n <= 0) {
        report(false, "BVH is not valid", valid, message, message_capacity);
        return LUX_OK;
    }
    Downloaded d;
    if (int st = download(ctx, bvh, d)) return st;
    std::string why = check_structure(d);
    if (!why.empty()) {
        report(false, why, valid, message, message_capacity);
        return LUX_OK;
    }
    if (bvh->n != n) {
        report(false, "BVH primitive count does not match scene primitive count", valid, message,
               message_capacity);
        return LUX_OK;
    }
    const size_t per = bvh->kind == LUX_PRIM_TRIANGLES ? 9 : 6;
    std::vector<float> host(per * size_t(n));
    cudaPointerAttributes attr{};
    bool on_device = cudaPointerGetAttributes(&attr, prims) == cudaSuccess &&
                     (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    if (on_device) {
        cudaError_t err = cudaMemcpy(host.data(), prims, sizeof(float) * host.size(),
                                     cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) return lux::cuda_fail(err, "primitive download");
    } else {
        std::memcpy(host.data(), prims, sizeof(float) * host.size());
    }
    std::vector<int> seen(n, 0);
    for (int k = 0; k < n; ++k) {
        int id = d.ids[k];
        if (id < 0 || id >= n) {
            report(false, "BVH contains primitive id not present in scene", valid, message,
                   message_capacity);
            return LUX_OK;
        }
        if (++seen[id] != 1) {
            report(false, "BVH contains duplicate primitive id", valid, message, message_capacity);
            return LUX_OK;
        }
        const float* p = &host[per * size_t(id)];
        HostBox want;
        if (per == 9) {
            for (int v = 0; v < 3; ++v)
                for (int a = 0; a < 3; ++a) {
                    want.lo[a] = std::fmin(want.lo[a], p[3 * v + a]);
                    want.hi[a] = std::fmax(want.hi[a], p[3 * v + a]);
                }
        } else {
            want = box_at(p);
        }
        if (!aabb_close(box_at(&d.bounds[6 * (size_t(n) - 1 + k)]), want)) {
            report(false, "BVH primitive bounds do not match scene primitive", valid, message,
                   message_capacity);
            return LUX_OK;
        }
    }
    report(true, "", valid, message, message_capacity);
    return LUX_OK;
}

}  // extern "C"
