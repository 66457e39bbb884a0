// The reference's GPU LBVH interface (bvh/gpu_bvh.cuh:25-61) and overlap queries
// (bvh/bvh_overlap.cuh:10-23) over liblux_gpu.so.  Replaces bvh/gpu_bvh.cu and
// bvh/bvh_overlap.cu; compiles against the reference's headers.
//
// GpuBvhStorage holds the library's BVH handle plus what the reference's interface needs
// beside it: the build input's primitive ids (the library numbers primitives by input
// position; the reference reports BvhBuildPrimitive::primitive_id) and the triangles last
// attached for ray queries, so that repeated queries with the same triangles upload them
// once per BVH.
//
// Results: build, refit and download give the reference host builder's codes, order,
// topology and boxes bit for bit; ray hits are the reference's stackless walk evaluated
// without contraction (its host arithmetic); overlap pair sets equal the reference's.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "bvh/bvh_overlap.cuh"
#include "bvh/gpu_bvh.cuh"

#include "lux_shim.h"

namespace lux_shim {

lux_ctx* context() {
    static lux_ctx* ctx = [] {
        lux_ctx* c = nullptr;
        check(lux_ctx_create(&c, 0, nullptr), "lux_ctx_create");
        return c;
    }();
    return ctx;
}

}  // namespace lux_shim

struct GpuBvhStorage {
    lux_bvh* bvh = nullptr;
    std::vector<int> ids;          // build input position -> BvhBuildPrimitive::primitive_id
    std::vector<float> attached;   // triangles last attached, 9 floats each, input order
    bool has_attached = false;
    ~GpuBvhStorage() {
        if (bvh) lux_bvh_destroy(bvh);
    }
};

namespace {

using lux_shim::check;
using lux_shim::context;

void append_box(std::vector<float>& out, const AABB& b) {
    out.insert(out.end(), {b.p_min.x, b.p_min.y, b.p_min.z, b.p_max.x, b.p_max.y, b.p_max.z});
}

void set_error(std::string* error_message, const std::string& message) {
    if (error_message) *error_message = message;
}

AABB box_at(const float* b) { return AABB(vec3(b[0], b[1], b[2]), vec3(b[3], b[4], b[5])); }

// The reference's own tolerance of the primitive-bounds check.
bool boxes_close(const AABB& a, const AABB& b) {
    const Float eps = Float(1e-4);
    return std::fabs(a.p_min.x - b.p_min.x) <= eps && std::fabs(a.p_min.y - b.p_min.y) <= eps
        && std::fabs(a.p_min.z - b.p_min.z) <= eps && std::fabs(a.p_max.x - b.p_max.x) <= eps
        && std::fabs(a.p_max.y - b.p_max.y) <= eps && std::fabs(a.p_max.z - b.p_max.z) <= eps;
}

// Overlap pairs from the library (input positions) as the reference reports them
// (primitive ids; self pairs with a < b).
OverlapQueryResult to_result(const std::vector<int32_t>& pairs, int64_t found, int max_pairs,
                             const std::vector<int>& left_ids, const std::vector<int>& right_ids,
                             bool self) {
    OverlapQueryResult res;
    res.found_count = static_cast<int>(found);
    res.truncated = found > max_pairs;
    const int64_t copy = std::min<int64_t>(found, max_pairs);
    res.pairs.reserve(static_cast<size_t>(copy));
    for (int64_t i = 0; i < copy; ++i) {
        int a = left_ids[pairs[2 * i]];
        int b = right_ids[pairs[2 * i + 1]];
        if (self && a > b) std::swap(a, b);
        res.pairs.push_back(PrimitivePair{a, b});
    }
    return res;
}

}  // namespace

GpuBvh::GpuBvh() : storage(std::make_unique<GpuBvhStorage>()) {}
GpuBvh::~GpuBvh() = default;
GpuBvh::GpuBvh(GpuBvh&& other) noexcept = default;
GpuBvh& GpuBvh::operator=(GpuBvh&& other) noexcept = default;

bool GpuBvh::is_valid() const {
    return storage && storage->bvh && primitive_count > 0 &&
           static_cast<int>(storage->ids.size()) == primitive_count;
}

// The library keeps its own node layouts (binary nodes with both child boxes and
// quantised 4-wide nodes); the reference's 32-byte stackless array is not materialised,
// so the view is empty.  Nothing on the B200 path reads it: the integrator shim renders
// through lux_render.
GpuBvhView GpuBvh::device_view() const { return GpuBvhView{}; }
const AABB* GpuBvh::overlap_bounds_device_ptr() const { return nullptr; }
const int* GpuBvh::overlap_primitive_ids_device_ptr() const { return nullptr; }
const uint32_t* GpuBvh::overlap_sorted_indices_device_ptr() const { return nullptr; }

GpuBvh build_gpu_lbvh(const std::vector<BvhBuildPrimitive>& primitives) {
    GpuBvh out;
    if (primitives.empty()) return out;
    std::vector<float> boxes;
    boxes.reserve(primitives.size() * 6);
    out.storage->ids.reserve(primitives.size());
    for (const BvhBuildPrimitive& p : primitives) {
        append_box(boxes, p.bounds);
        out.storage->ids.push_back(p.primitive_id);
    }
    const int n = static_cast<int>(primitives.size());
    check(lux_lbvh_build(context(), boxes.data(), n, LUX_PRIM_AABBS, 30, &out.storage->bvh),
          "build_gpu_lbvh");
    float root[6];
    check(lux_bvh_info(context(), out.storage->bvh, nullptr, nullptr, nullptr, root),
          "build_gpu_lbvh");
    out.root_bounds = box_at(root);
    out.primitive_count = n;
    return out;
}

bool refit_gpu_lbvh(GpuBvh& bvh, const std::vector<BvhBuildPrimitive>& primitives) {
    if (!bvh.is_valid() || static_cast<int>(primitives.size()) != bvh.primitive_count)
        return false;
    std::vector<float> boxes;
    boxes.reserve(primitives.size() * 6);
    for (size_t i = 0; i < primitives.size(); ++i) {
        if (primitives[i].primitive_id != bvh.storage->ids[i]) return false;
        append_box(boxes, primitives[i].bounds);
    }
    int st = lux_lbvh_refit(context(), bvh.storage->bvh, boxes.data(), bvh.primitive_count);
    if (st == LUX_ERR_MISMATCH) return false;
    check(st, "refit_gpu_lbvh");
    float root[6];
    check(lux_bvh_info(context(), bvh.storage->bvh, nullptr, nullptr, nullptr, root),
          "refit_gpu_lbvh");
    bvh.root_bounds = box_at(root);
    bvh.storage->has_attached = false;  // the triangles no longer match the new boxes
    return true;
}

CpuBvhTree download_bvh_for_validation(const GpuBvh& bvh) {
    CpuBvhTree tree;
    if (!bvh.is_valid()) return tree;
    const int n = bvh.primitive_count;
    const int nodes = 2 * n - 1;
    std::vector<int32_t> sorted(n), left(nodes), right(nodes);
    std::vector<float> bounds(size_t(nodes) * 6);
    check(lux_bvh_download(context(), bvh.storage->bvh, nullptr, sorted.data(), left.data(),
                           right.data(), bounds.data()),
          "download_bvh_for_validation");
    tree.root_node = 0;
    tree.nodes.resize(nodes);
    tree.primitive_ids.reserve(n);
    for (int i = 0; i < nodes; ++i) {
        CpuBvhNode& node = tree.nodes[i];
        node.bounds = box_at(&bounds[size_t(i) * 6]);
        node.left = left[i];
        node.right = right[i];
    }
    for (int k = 0; k < n; ++k) {
        CpuBvhNode& leaf = tree.nodes[n - 1 + k];
        leaf.left = leaf.right = -1;
        leaf.first_primitive = k;
        leaf.primitive_count = 1;
        tree.primitive_ids.push_back(bvh.storage->ids[sorted[k]]);
    }
    return tree;
}

bool validate_gpu_bvh_structure(const GpuBvh& bvh, std::string* error_message) {
    if (!bvh.is_valid()) {
        set_error(error_message, "BVH is not valid");
        return false;
    }
    int32_t valid = 0;
    char message[512] = {};
    check(lux_bvh_validate_structure(context(), bvh.storage->bvh, &valid, message,
                                     sizeof(message)),
          "validate_gpu_bvh_structure");
    if (!valid) set_error(error_message, message);
    return valid != 0;
}

bool validate_gpu_bvh_matches_primitives(const GpuBvh& bvh,
                                         const std::vector<BvhBuildPrimitive>& primitives,
                                         std::string* error_message) {
    if (primitives.empty()) {
        if (!bvh.is_valid() && bvh.primitive_count == 0) return true;
        set_error(error_message, "BVH contains primitives for an empty scene");
        return false;
    }
    std::string structure_error;
    if (!validate_gpu_bvh_structure(bvh, &structure_error)) {
        set_error(error_message,
                  structure_error.empty() ? "BVH structure validation failed" : structure_error);
        return false;
    }
    if (bvh.primitive_count != static_cast<int>(primitives.size())) {
        set_error(error_message, "BVH primitive count does not match scene primitive count");
        return false;
    }
    std::unordered_map<int, const BvhBuildPrimitive*> expected;
    expected.reserve(primitives.size());
    for (const BvhBuildPrimitive& p : primitives) {
        if (!expected.emplace(p.primitive_id, &p).second) {
            set_error(error_message, "Scene primitive ids are not unique");
            return false;
        }
    }
    // Every leaf's box is its build input's box, downloaded in sorted order.
    CpuBvhTree tree = download_bvh_for_validation(bvh);
    const int n = bvh.primitive_count;
    std::unordered_map<int, int> seen;
    seen.reserve(primitives.size());
    for (int k = 0; k < n; ++k) {
        int id = tree.primitive_ids[k];
        auto it = expected.find(id);
        if (it == expected.end()) {
            set_error(error_message, "BVH contains primitive id not present in scene");
            return false;
        }
        if (++seen[id] != 1) {
            set_error(error_message, "BVH contains duplicate primitive id");
            return false;
        }
        if (!boxes_close(tree.nodes[n - 1 + k].bounds, it->second->bounds)) {
            set_error(error_message, "BVH primitive bounds do not match scene primitive");
            return false;
        }
    }
    if (seen.size() != expected.size()) {
        set_error(error_message, "BVH is missing one or more scene primitives");
        return false;
    }
    return true;
}

std::vector<GpuRayHit> intersect_gpu_bvh_stackless(const GpuBvh& bvh,
                                                   const std::vector<Triangle>& triangles,
                                                   const std::vector<Ray>& rays) {
    std::vector<GpuRayHit> hits(rays.size());
    if (!bvh.is_valid() || rays.empty()) return hits;
    GpuBvhStorage& s = *bvh.storage;
    const int n = bvh.primitive_count;
    // triangles is indexed by primitive id (as the reference's kernel reads it); the
    // library wants them in build input order.
    std::vector<float> soup(size_t(n) * 9);
    for (int i = 0; i < n; ++i) {
        const int id = s.ids[i];
        if (id < 0 || id >= static_cast<int>(triangles.size()))
            throw std::runtime_error("intersect_gpu_bvh_stackless: primitive id outside triangles");
        const Triangle& t = triangles[id];
        const float v[9] = {t.v0.x, t.v0.y, t.v0.z, t.v1.x, t.v1.y, t.v1.z, t.v2.x, t.v2.y, t.v2.z};
        std::memcpy(&soup[size_t(i) * 9], v, sizeof(v));
    }
    if (!s.has_attached || s.attached != soup) {
        check(lux_bvh_attach_triangles(context(), s.bvh, soup.data(), n),
              "intersect_gpu_bvh_stackless");
        s.attached.swap(soup);
        s.has_attached = true;
    }
    std::vector<float> r;
    r.reserve(rays.size() * 8);
    for (const Ray& ray : rays)
        r.insert(r.end(), {ray.origin.x, ray.origin.y, ray.origin.z, ray.t_min,
                           ray.direction.x, ray.direction.y, ray.direction.z, ray.t_max});
    std::vector<int32_t> id(rays.size());
    std::vector<float> t(rays.size());
    check(lux_trace_closest(context(), s.bvh, r.data(), static_cast<int32_t>(rays.size()),
                            id.data(), t.data()),
          "intersect_gpu_bvh_stackless");
    for (size_t i = 0; i < rays.size(); ++i)
        hits[i] = id[i] >= 0 ? GpuRayHit{s.ids[id[i]], t[i]} : GpuRayHit{-1, INFINITY};
    return hits;
}

OverlapQueryResult query_aabb_overlaps_self(const GpuBvh& bvh, int max_pairs) {
    if (!bvh.is_valid() || max_pairs <= 0) return OverlapQueryResult{};
    std::vector<int32_t> pairs(size_t(max_pairs) * 2);
    int64_t found = 0;
    check(lux_overlap_self(context(), bvh.storage->bvh, pairs.data(), max_pairs, &found),
          "query_aabb_overlaps_self");
    return to_result(pairs, found, max_pairs, bvh.storage->ids, bvh.storage->ids, true);
}

OverlapQueryResult query_aabb_overlaps_cross(const GpuBvh& left, const GpuBvh& right,
                                             int max_pairs) {
    if (!left.is_valid() || !right.is_valid() || max_pairs <= 0) return OverlapQueryResult{};
    std::vector<int32_t> pairs(size_t(max_pairs) * 2);
    int64_t found = 0;
    check(lux_overlap_cross(context(), left.storage->bvh, right.storage->bvh, pairs.data(),
                            max_pairs, &found),
          "query_aabb_overlaps_cross");
    return to_result(pairs, found, max_pairs, left.storage->ids, right.storage->ids, false);
}
