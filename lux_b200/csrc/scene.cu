// Scene upload for the path tracer: world-space triangles, BLAS per mesh, TLAS over
// instances, materials and light tables.
//
// Host arithmetic restates the reference's host preparation so that every uploaded
// value is bit-identical to what the reference computes (paths relative to src/):
//   transform_point / transform_normal / transform_bounds   core/mat4.cuh:173-275
//   inverse_affine                                          core/mat4.cuh:131-160
//   scene triangle order (instances, then local triangles)  scene/scene_data.h:282-329
//   prepare_scene_light_sampling (area + explicit lights)   scene/scene_prepare.h:268-387
//   build_alias_table_from_weights                          light/light_distribution.cpp:8-61
//   build_light_bvh (the light tree)                        light/light_distribution.cpp:68-161
// The host compiler evaluates these without contraction (x86-64 baseline ISA).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/lux_gpu.h"
#include "pt_scene.h"

namespace lux {
namespace {

using pt::AliasEntry;
using pt::Instance;
using pt::Light;
using pt::Material;

// The helpers below run on the host and, for device-side preparation, on the device:
// this file is compiled without contraction and with IEEE division and square root, so
// both sides round every operation alike.
#define SCENE_HD __host__ __device__

struct V3 {
    float x, y, z;
};
SCENE_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
SCENE_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
SCENE_HD float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SCENE_HD V3 cross3(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
SCENE_HD float len3(V3 a) { return sqrtf(dot3(a, a)); }
SCENE_HD V3 normalize3(V3 v) {
    float l = len3(v);
    if (!(l > 0)) return v;
    float inv = 1.0f / l;
    return v3(v.x * inv, v.y * inv, v.z * inv);
}

// transform_point (core/mat4.cuh:173-184) on a row-major 3x4 affine matrix.
SCENE_HD V3 transform_point(const float* m, V3 p) {
    float x = m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3];
    float y = m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7];
    float z = m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11];
    float w = 0.0f * p.x + 0.0f * p.y + 0.0f * p.z + 1.0f;
    return w == 1 ? v3(x, y, z) : v3(x / w, y / w, z / w);
}

// transform_normal (core/mat4.cuh:207-230): adjugate-transpose, then normalize.
SCENE_HD V3 transform_normal(const float* m, V3 n) {
    float a00 = m[5] * m[10] - m[6] * m[9];
    float a01 = m[6] * m[8] - m[4] * m[10];
    float a02 = m[4] * m[9] - m[5] * m[8];
    float a10 = m[2] * m[9] - m[1] * m[10];
    float a11 = m[0] * m[10] - m[2] * m[8];
    float a12 = m[1] * m[8] - m[0] * m[9];
    float a20 = m[1] * m[6] - m[2] * m[5];
    float a21 = m[2] * m[4] - m[0] * m[6];
    float a22 = m[0] * m[5] - m[1] * m[4];
    V3 t = v3(a00 * n.x + a01 * n.y + a02 * n.z, a10 * n.x + a11 * n.y + a12 * n.z,
              a20 * n.x + a21 * n.y + a22 * n.z);
    return normalize3(t);
}

// transform_instance_normal (scene/scene_data.h:223-229).
SCENE_HD V3 instance_normal(const float* m, V3 n) {
    if (dot3(n, n) == 0) return v3(0, 0, 0);
    V3 t = transform_normal(m, n);
    if (dot3(t, t) == 0) return v3(0, 0, 0);
    return normalize3(t);
}

// inverse_affine (core/mat4.cuh:131-160).
void inverse_affine(const float* m, float* r) {
    float a00 = m[0], a01 = m[1], a02 = m[2];
    float a10 = m[4], a11 = m[5], a12 = m[6];
    float a20 = m[8], a21 = m[9], a22 = m[10];
    float det = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20)
              + a02 * (a10 * a21 - a11 * a20);
    for (int i = 0; i < 12; ++i) r[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    if (std::fabs(det) <= 1e-12f) return;
    float inv_det = 1.0f / det;
    r[0] = (a11 * a22 - a12 * a21) * inv_det;
    r[1] = -(a01 * a22 - a02 * a21) * inv_det;
    r[2] = (a01 * a12 - a02 * a11) * inv_det;
    r[4] = -(a10 * a22 - a12 * a20) * inv_det;
    r[5] = (a00 * a22 - a02 * a20) * inv_det;
    r[6] = -(a00 * a12 - a02 * a10) * inv_det;
    r[8] = (a10 * a21 - a11 * a20) * inv_det;
    r[9] = -(a00 * a21 - a01 * a20) * inv_det;
    r[10] = (a00 * a11 - a01 * a10) * inv_det;
    float tx = m[3], ty = m[7], tz = m[11];
    r[3] = -(r[0] * tx + r[1] * ty + r[2] * tz);
    r[7] = -(r[4] * tx + r[5] * ty + r[6] * tz);
    r[11] = -(r[8] * tx + r[9] * ty + r[10] * tz);
}

float luminance(V3 v) { return 0.2126f * v.x + 0.7152f * v.y + 0.0722f * v.z; }

struct Box {
    V3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
    void expand(V3 p) {
        lo = v3(std::fmin(lo.x, p.x), std::fmin(lo.y, p.y), std::fmin(lo.z, p.z));
        hi = v3(std::fmax(hi.x, p.x), std::fmax(hi.y, p.y), std::fmax(hi.z, p.z));
    }
    bool empty() const { return lo.x > hi.x || lo.y > hi.y || lo.z > hi.z; }
};

// build_alias_table_from_weights (light/light_distribution.cpp:8-61).
std::vector<AliasEntry> alias_from_weights(const std::vector<float>& weights) {
    int count = static_cast<int>(weights.size());
    std::vector<AliasEntry> table(count);
    if (count <= 0) return table;
    float total = 0;
    for (float w : weights) total += std::fmax(0.0f, w);
    if (total <= 0) return {};
    std::vector<float> scaled(count, 0);
    std::vector<int> small, large;
    for (int i = 0; i < count; ++i) {
        float pmf = std::fmax(0.0f, weights[i]) / total;
        table[i].pmf = pmf;
        table[i].alias = i;
        table[i].probability = 1.0f;
        scaled[i] = pmf * static_cast<float>(count);
        if (scaled[i] < 1.0f) small.push_back(i);
        else large.push_back(i);
    }
    while (!small.empty() && !large.empty()) {
        int less = small.back();
        small.pop_back();
        int more = large.back();
        large.pop_back();
        table[less].probability = scaled[less];
        table[less].alias = more;
        scaled[more] = (scaled[more] + scaled[less]) - 1.0f;
        if (scaled[more] < 1.0f) small.push_back(more);
        else large.push_back(more);
    }
    for (int i : large) { table[i].probability = 1.0f; table[i].alias = i; }
    for (int i : small) { table[i].probability = 1.0f; table[i].alias = i; }
    return table;
}

// ---- light tree (build_light_bvh, light/light_distribution.cpp:68-161)

struct LightItem {  // LightBvhBuildItem (light/light_distribution.h:42-47)
    Box box;
    V3 centroid;
    int light;
    float power;
};

V3 centre(const Box& b) {  // AABB::centroid
    return v3((b.lo.x + b.hi.x) * 0.5f, (b.lo.y + b.hi.y) * 0.5f, (b.lo.z + b.hi.z) * 0.5f);
}

struct LightTree {
    std::vector<pt::LightNode> nodes;   // preorder, the root first
    std::vector<int> leaf;              // light index -> leaf node, -1 outside the tree
    std::vector<int> other_slot;        // light index -> slot of other_lights, -1 none
    std::vector<int> other_lights;      // the lights outside the tree with a positive weight
    std::vector<AliasEntry> other_alias;
    float other_power = 0;
};

float axis_of(const V3& v, int axis) { return axis == 0 ? v.x : axis == 1 ? v.y : v.z; }

// Nodes for items[begin, end): a leaf per light; otherwise a median split on the widest
// axis of the centroids' box, the median placed by std::nth_element with the reference's
// comparison, so that the same items in the same order give the same tree.  An internal
// node holds the union of its children's boxes and the sum of their powers.
int light_tree_range(std::vector<LightItem>& items, int begin, int end, int parent,
                     LightTree& t) {
    const int index = static_cast<int>(t.nodes.size());
    t.nodes.push_back(pt::LightNode{});
    pt::LightNode node{};
    node.parent = parent;
    node.left = node.right = -1;
    if (end - begin == 1) {
        const LightItem& it = items[begin];
        node.lo = make_f3(it.box.lo.x, it.box.lo.y, it.box.lo.z);
        node.hi = make_f3(it.box.hi.x, it.box.hi.y, it.box.hi.z);
        node.power = it.power;
        node.light = it.light;
        t.leaf[it.light] = index;
        t.nodes[index] = node;
        return index;
    }
    Box centroids;
    for (int i = begin; i < end; ++i) centroids.expand(items[i].centroid);
    const V3 d = v3(centroids.hi.x - centroids.lo.x, centroids.hi.y - centroids.lo.y,
                    centroids.hi.z - centroids.lo.z);
    const int axis = (d.x > d.y && d.x > d.z) ? 0 : (d.y > d.z) ? 1 : 2;  // max_extent_axis
    const int mid = begin + (end - begin) / 2;
    std::nth_element(items.begin() + begin, items.begin() + mid, items.begin() + end,
                     [axis](const LightItem& a, const LightItem& b) {
                         return axis_of(a.centroid, axis) < axis_of(b.centroid, axis);
                     });
    const int left = light_tree_range(items, begin, mid, index, t);
    const int right = light_tree_range(items, mid, end, index, t);
    const pt::LightNode& l = t.nodes[left];
    const pt::LightNode& r = t.nodes[right];
    node.left = left;
    node.right = right;
    node.light = -1;
    node.power = l.power + r.power;
    node.lo = make_f3(std::fmin(l.lo.x, r.lo.x), std::fmin(l.lo.y, r.lo.y), std::fmin(l.lo.z, r.lo.z));
    node.hi = make_f3(std::fmax(l.hi.x, r.hi.x), std::fmax(l.hi.y, r.hi.y), std::fmax(l.hi.z, r.hi.z));
    t.nodes[index] = node;
    return index;
}

// The tree over items (lights with bounds, in light-index order) and the power table of
// the other lights, their weights taken from the selection table's running sums cdf.
LightTree build_light_tree(std::vector<LightItem> items, const std::vector<float>& cdf) {
    LightTree t;
    const int count = static_cast<int>(cdf.size());
    if (items.empty() || count == 0) return t;
    std::vector<char> seen(count, 0);
    for (const LightItem& it : items) seen[it.light] = 1;
    t.other_slot.assign(count, -1);
    std::vector<float> other_cdf;
    float other_weight = 0;
    for (int i = 0; i < count; ++i) {
        if (seen[i]) continue;
        const float w = cdf[i] - (i == 0 ? 0.0f : cdf[i - 1]);
        if (w <= 0) continue;
        other_weight += w;
        t.other_slot[i] = static_cast<int>(t.other_lights.size());
        t.other_lights.push_back(i);
        other_cdf.push_back(other_weight);
    }
    t.other_power = other_weight;
    if (!other_cdf.empty() && other_weight > 0) {  // build_alias_table_from_cdf
        std::vector<float> w;
        float prev = 0;
        for (float c : other_cdf) {
            w.push_back(c - prev);
            prev = c;
        }
        t.other_alias = alias_from_weights(w);
    }
    t.leaf.assign(count, -1);
    t.nodes.reserve(items.size() * 2 - 1);
    light_tree_range(items, 0, static_cast<int>(items.size()), -1, t);
    return t;
}

// ---- light tables (prepare_scene_light_sampling, scene/scene_prepare.h:268-387)

struct LightTables {
    std::vector<Light> lights;
    std::vector<float> cdf;              // running power sums
    float total = 0;
    int area_count = 0;
    std::vector<int> primitive_light;    // scene triangle -> light (-1 none, -2 several)
    std::vector<AliasEntry> alias;       // power alias table
    LightTree tree;
};

// Area lights from the emissive triangles (scene order; a triangle without area is no
// light), then the explicit lights with their powers; the power alias table; the tree
// over the lights with bounds (area lights: their triangle's box; point lights: their
// position; light_bounds_for_bvh, scene/scene_prepare.h:243-296).
LightTables make_light_tables(const std::vector<lux_scene::EmissiveTri>& emissive,
                              const std::vector<Light>& explicit_lights,
                              const std::vector<float>& explicit_power, size_t triangle_count) {
    LightTables t;
    t.primitive_light.assign(triangle_count, -1);
    std::vector<float> power;
    std::vector<Box> boxes;
    auto append = [&](const Light& l, float p, const Box& b) -> int {
        if (p <= 0) return -1;
        t.total += p;
        t.lights.push_back(l);
        t.cdf.push_back(t.total);
        power.push_back(p);
        boxes.push_back(b);
        return static_cast<int>(t.lights.size()) - 1;
    };
    for (const lux_scene::EmissiveTri& e : emissive) {
        const V3 a = v3(e.w[0], e.w[1], e.w[2]);
        const V3 b = v3(e.w[3], e.w[4], e.w[5]);
        const V3 c = v3(e.w[6], e.w[7], e.w[8]);
        const float area = 0.5f * len3(cross3(b - a, c - a));
        if (area <= 0) continue;
        Light l;
        l.kind = 0;
        l.primitive = e.triangle;
        l.two_sided = e.two_sided;
        l.area = area;
        l.emission = make_f3(e.emission[0], e.emission[1], e.emission[2]);
        l.vec = make_f3(0, 0, 0);
        l.image = e.image;
        l.image_scale = make_f3(e.image_scale[0], e.image_scale[1], e.image_scale[2]);
        Box box;
        box.expand(a);
        box.expand(b);
        box.expand(c);
        const float p = area * std::fmax(1e-6f, e.power_hint);
        const int index = append(l, p, box);
        if (index >= 0) {
            int& stored = t.primitive_light[e.triangle];
            stored = stored == -1 ? index : -2;
        }
    }
    t.area_count = static_cast<int>(t.lights.size());
    for (size_t i = 0; i < explicit_lights.size(); ++i) {
        const Light& l = explicit_lights[i];
        Box box;  // empty: no place in the tree
        if (l.kind == 1) box.lo = box.hi = v3(l.vec.x, l.vec.y, l.vec.z);
        append(l, explicit_power[i], box);
    }
    if (t.total > 0) {  // finalize_light_selection_table
        std::vector<float> weights;
        float prev = 0;
        for (float c : t.cdf) {
            weights.push_back(c - prev);
            prev = c;
        }
        t.alias = alias_from_weights(weights);
    }
    std::vector<LightItem> items;
    for (int i = 0; i < static_cast<int>(t.lights.size()); ++i)
        if (!boxes[i].empty()) items.push_back(LightItem{boxes[i], centre(boxes[i]), i, power[i]});
    t.tree = build_light_tree(items, t.cdf);
    return t;
}

template <typename T>
int upload(T** dst, const std::vector<T>& src, cudaStream_t stream) {
    size_t bytes = sizeof(T) * std::max<size_t>(src.size(), 1);
    cudaError_t err = cudaMalloc(reinterpret_cast<void**>(dst), bytes);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return fail(LUX_ERR_OUT_OF_MEMORY, "scene allocation failed");
    }
    if (!src.empty()) {
        err = cudaMemcpyAsync(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice,
                              stream);
        if (err != cudaSuccess) return cuda_fail(err, "scene upload");
    }
    return LUX_OK;
}

// Copies src into *dst, in stream order when it fits the buffer's capacity; otherwise
// waits for the stream once (earlier work may still read the old buffer), then
// reallocates.
template <typename T>
int refill(T** dst, size_t* capacity, const std::vector<T>& src, cudaStream_t stream,
           bool* synced) {
    if (!*dst || src.size() > *capacity) {
        if (*dst) {
            if (!*synced) {
                cudaError_t err = cudaStreamSynchronize(stream);
                if (err != cudaSuccess) return cuda_fail(err, "light table update");
                *synced = true;
            }
            cudaFree(*dst);
            *dst = nullptr;
        }
        *capacity = std::max<size_t>(src.size(), 1);
        if (cudaMalloc(reinterpret_cast<void**>(dst), sizeof(T) * *capacity) != cudaSuccess) {
            cudaGetLastError();
            *dst = nullptr;
            *capacity = 0;
            return fail(LUX_ERR_OUT_OF_MEMORY, "scene allocation failed");
        }
    }
    if (src.empty()) return LUX_OK;
    cudaError_t err = cudaMemcpyAsync(*dst, src.data(), sizeof(T) * src.size(),
                                      cudaMemcpyHostToDevice, stream);
    return err == cudaSuccess ? LUX_OK : cuda_fail(err, "scene upload");
}

int upload_light_tables(lux_ctx* ctx, lux_scene* s, const LightTables& t) {
    cudaStream_t stream = ctx->stream;
    lux_scene::LightCapacity& c = s->light_capacity;
    bool synced = false;
    int st = refill(&s->lights, &c.lights, t.lights, stream, &synced);
    if (!st) st = refill(&s->light_alias, &c.alias, t.alias, stream, &synced);
    if (!st) st = refill(&s->primitive_light, &c.primitive, t.primitive_light, stream, &synced);
    if (!st && !t.tree.nodes.empty()) {
        st = refill(&s->light_tree, &c.tree, t.tree.nodes, stream, &synced);
        if (!st) st = refill(&s->light_leaf, &c.leaf, t.tree.leaf, stream, &synced);
        if (!st) st = refill(&s->light_other_slot, &c.other_slot, t.tree.other_slot, stream, &synced);
        if (!st) st = refill(&s->other_lights, &c.other_lights, t.tree.other_lights, stream, &synced);
        if (!st) st = refill(&s->other_alias, &c.other_alias, t.tree.other_alias, stream, &synced);
    }
    return st;
}

void set_light_view(lux_scene* s, const LightTables& t) {
    pt::SceneView& v = s->view;
    const bool tree = !t.tree.nodes.empty();
    v.lights = s->lights;
    v.light_count = static_cast<int>(t.lights.size());
    v.total_light_power = t.total;
    v.light_alias = t.alias.empty() ? nullptr : s->light_alias;
    v.light_sampler = 1;
    v.primitive_light = s->primitive_light;
    v.light_tree = tree ? s->light_tree : nullptr;
    v.light_tree_count = static_cast<int>(t.tree.nodes.size());
    v.light_tree_root = tree ? 0 : -1;
    v.light_leaf = tree ? s->light_leaf : nullptr;
    v.light_other_slot = tree ? s->light_other_slot : nullptr;
    v.other_lights = tree && !t.tree.other_lights.empty() ? s->other_lights : nullptr;
    v.other_alias = tree && !t.tree.other_alias.empty() ? s->other_alias : nullptr;
    v.other_count = static_cast<int>(t.tree.other_lights.size());
    v.other_power = t.tree.other_power;
    s->area_light_count = t.area_count;
}

Material to_material(const lux_material& m) {
    Material r;
    r.type = m.type;
    r.albedo = make_f3(m.albedo[0], m.albedo[1], m.albedo[2]);
    r.emission = make_f3(m.emission[0], m.emission[1], m.emission[2]);
    r.two_sided = m.emission_two_sided ? 1 : 0;
    r.roughness = m.roughness;
    r.metallic = m.metallic;
    r.eta = m.eta;
    r.emission_image = m.emission_source == 1 ? m.emission_image : -1;
    r.emission_scale = make_f3(m.emission_scale[0], m.emission_scale[1], m.emission_scale[2]);
    return r;
}

// Material::is_emissive (material/material.h:104-108).
bool is_emissive(const lux_material& m) {
    return std::fmax(m.emission[0], std::fmax(m.emission[1], m.emission[2])) > 0 ||
           (m.emission_source == 1 && m.emission_image >= 0);
}

// scene_material_emission_power_hint (scene/scene_data.h:189-205): the luminance of the
// emission, or the mean luminance of the scaled texels of an emission image.
float emission_power_hint(const lux_scene_desc* d, const lux_material& m) {
    if (m.emission_source != 1) return luminance(v3(m.emission[0], m.emission[1], m.emission[2]));
    const lux_env_image& im = d->images[m.emission_image];
    const size_t count = size_t(im.width) * size_t(im.height);
    float sum = 0;
    for (size_t i = 0; i < count; ++i) {
        const float* p = im.pixels + 3 * i;
        sum += luminance(v3(p[0] * m.emission_scale[0], p[1] * m.emission_scale[1],
                            p[2] * m.emission_scale[2]));
    }
    return sum / static_cast<float>(count);
}

// ---- device-side preparation

constexpr int kPrepThreads = 256;

// One mesh's device arrays (slices of the scene's concatenated mesh buffers).
struct MeshDev {
    const float* vertices;      // 3 per vertex
    const float* normals;       // 3 per vertex, or null
    const float* uvs;           // 2 per vertex, or null
    const uint32_t* indices;    // 3 per triangle
    const int32_t* material_ids;
    int triangle_count;
};

// World triangle and shading record of every scene triangle (scene order: instances,
// then local triangles; scene/scene_data.h:282-329): transform_point of the corners,
// transform_instance_normal of the corner normals, the corner texcoords, and the tags
// (material, instance, local triangle) in the .w lanes.  A triangle uses its normals
// only when all three are nonzero after the transform.
__global__ void k_world_triangles(const MeshDev* meshes, const Instance* instances,
                                  const int* overrides, int instance_count, int total,
                                  pt::SceneTri* tris, pt::SceneTriShading* shading) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
        int lo = 0, hi = instance_count - 1;  // the last instance starting at or before p
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (instances[mid].first_primitive <= p) lo = mid;
            else hi = mid - 1;
        }
        const Instance& inst = instances[lo];
        const int t = p - inst.first_primitive;
        const MeshDev& mesh = meshes[inst.blas];
        V3 w[3], n[3];
        float uv[3][2] = {{0, 0}, {0, 0}, {0, 0}};
        bool has_normals = mesh.normals != nullptr;
        for (int k = 0; k < 3; ++k) {
            const uint32_t v = mesh.indices[3 * size_t(t) + k];
            const float* q = mesh.vertices + 3 * size_t(v);
            w[k] = transform_point(inst.m, v3(q[0], q[1], q[2]));
            if (mesh.normals) {
                const float* r = mesh.normals + 3 * size_t(v);
                n[k] = instance_normal(inst.m, v3(r[0], r[1], r[2]));
                if (dot3(n[k], n[k]) <= 0) has_normals = false;
            } else {
                n[k] = v3(0, 0, 0);
            }
            if (mesh.uvs) {
                uv[k][0] = mesh.uvs[2 * size_t(v)];
                uv[k][1] = mesh.uvs[2 * size_t(v) + 1];
            }
        }
        const int material = overrides[lo] >= 0 ? overrides[lo] : mesh.material_ids[t];
        pt::SceneTri st;
        st.v0 = make_float4(w[0].x, w[0].y, w[0].z, __int_as_float(material));
        st.v1 = make_float4(w[1].x, w[1].y, w[1].z, __int_as_float(lo));
        st.v2 = make_float4(w[2].x, w[2].y, w[2].z, __int_as_float(t));
        tris[p] = st;
        pt::SceneTriShading sh;
        sh.n0 = make_float4(n[0].x, n[0].y, n[0].z, uv[0][0]);
        sh.n1 = make_float4(n[1].x, n[1].y, n[1].z, uv[0][1]);
        sh.n2 = make_float4(n[2].x, n[2].y, n[2].z, uv[1][0]);
        sh.uv = make_float4(uv[1][1], uv[2][0], uv[2][1], has_normals ? 1.0f : 0.0f);
        shading[p] = sh;
    }
}

__global__ void k_mesh_soup(const float* vertices, int vertex_count, const uint32_t* indices,
                            int triangle_count, float* soup, int* error);

// TLAS entry boxes at creation: transform_bounds (core/mat4.cuh:259-275) of each entry's
// mesh box, the root box of the mesh's BLAS (the union of its triangle boxes,
// finalize_scene_mesh, scene/scene_data.h:215-220).
__global__ void k_tlas_boxes(const Instance* instances, const int* tlas_instance,
                             const BvhView* blas, int entry_count, float* boxes) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= entry_count) return;
    const Instance& inst = instances[tlas_instance[k]];
    const float* r = blas[inst.blas].root;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (!(r[0] > r[3] || r[1] > r[4] || r[2] > r[5])) {
        for (int c = 0; c < 8; ++c) {
            const V3 w = transform_point(inst.m, v3((c & 1) ? r[3] : r[0], (c & 2) ? r[4] : r[1],
                                                    (c & 4) ? r[5] : r[2]));
            lo[0] = fminf(lo[0], w.x); lo[1] = fminf(lo[1], w.y); lo[2] = fminf(lo[2], w.z);
            hi[0] = fmaxf(hi[0], w.x); hi[1] = fmaxf(hi[1], w.y); hi[2] = fmaxf(hi[2], w.z);
        }
    }
    for (int a = 0; a < 3; ++a) {
        boxes[6 * k + a] = lo[a];
        boxes[6 * k + 3 + a] = hi[a];
    }
}

int prep_blocks(lux_ctx* ctx, int64_t items) {
    const int64_t b = (items + kPrepThreads - 1) / kPrepThreads;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, int64_t(ctx->sm_count) * 16)));
}

}  // namespace

void scene_free(lux_scene* s) {
    for (auto& r : s->refit) {
        cudaFree(r.vertices);
        cudaFree(r.indices);
        cudaFree(r.instances);
    }
    s->refit.clear();
    void* ptrs[] = {s->materials, s->tris, s->shading, s->d_instances, s->tlas_instance,
                    s->blas_views, s->lights, s->light_alias, s->primitive_light, s->tri_soup,
                    s->tlas_boxes, s->env_pixels, s->env_cdf, s->d_env, s->light_tree,
                    s->mesh_data.vertices, s->mesh_data.normals, s->mesh_data.uvs,
                    s->mesh_data.indices, s->mesh_data.material_ids, s->image_pixels,
                    s->d_images,
                    s->light_leaf, s->light_other_slot, s->other_lights, s->other_alias};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (lux_bvh* b : s->blas) lux_bvh_destroy(b);
    if (s->tlas) lux_bvh_destroy(s->tlas);
    s->blas.clear();
    s->tlas = nullptr;
}

int scene_create(lux_ctx* ctx, const lux_scene_desc* d, lux_scene** out) {
    if (d->material_count < 0 || d->mesh_count < 0 || d->instance_count < 0 || d->light_count < 0)
        return fail(LUX_ERR_INVALID_ARGUMENT, "negative scene counts");
    for (int i = 0; i < d->mesh_count; ++i) {
        const lux_mesh_desc& m = d->meshes[i];
        if (m.triangle_count < 0 || m.vertex_count < 0 || (m.triangle_count > 0 &&
            (!m.indices || !m.vertices || !m.material_ids)))
            return fail(LUX_ERR_INVALID_ARGUMENT, "bad mesh description");
        for (int t = 0; t < 3 * m.triangle_count; ++t)
            if (m.indices[t] >= static_cast<uint32_t>(m.vertex_count))
                return fail(LUX_ERR_INVALID_ARGUMENT, "mesh index out of range");
        for (int t = 0; t < m.triangle_count; ++t)
            if (m.material_ids[t] < 0 || m.material_ids[t] >= d->material_count)
                return fail(LUX_ERR_INVALID_ARGUMENT, "material id out of range");
    }
    for (int i = 0; i < d->material_count; ++i) {
        if (d->materials[i].type < 0 || d->materials[i].type > 5)
            return fail(LUX_ERR_INVALID_ARGUMENT, "unknown material type");
        const lux_material& m = d->materials[i];
        if (m.emission_source < 0 || m.emission_source > 1)
            return fail(LUX_ERR_INVALID_ARGUMENT, "unknown emission source");
        if (m.emission_source == 1 &&
            (m.emission_image < 0 || m.emission_image >= d->image_count || !d->images))
            return fail(LUX_ERR_INVALID_ARGUMENT, "image emission without a valid image");
    }
    for (int i = 0; i < d->image_count; ++i) {
        const lux_env_image& e = d->images[i];
        if (!e.pixels || e.width <= 0 || e.height <= 0 ||
            static_cast<long long>(e.width) * e.height > (1ll << 26))
            return fail(LUX_ERR_INVALID_ARGUMENT, "bad scene image");
    }
    for (int i = 0; i < d->instance_count; ++i) {
        const lux_instance_desc& in = d->instances[i];
        if (in.mesh < 0 || in.mesh >= d->mesh_count)
            return fail(LUX_ERR_INVALID_ARGUMENT, "instance mesh out of range");
        if (in.material_override >= d->material_count)
            return fail(LUX_ERR_INVALID_ARGUMENT, "instance material out of range");
    }
    for (int i = 0; i < d->light_count; ++i) {
        if (d->lights[i].kind < 1 || d->lights[i].kind > 4)
            return fail(LUX_ERR_INVALID_ARGUMENT, "unknown light kind");
        if (d->lights[i].kind == 4) {
            const int im = d->lights[i].image;
            if (im < 0 || im >= d->image_count || !d->images)
                return fail(LUX_ERR_INVALID_ARGUMENT, "image light without a valid image");
            const lux_env_image& e = d->images[im];
            if (!e.pixels || e.width <= 0 || e.height <= 0 ||
                static_cast<long long>(e.width) * e.height > (1ll << 26))
                return fail(LUX_ERR_INVALID_ARGUMENT, "bad environment image");
        }
    }

    lux_scene* s = new (std::nothrow) lux_scene();
    if (!s) return fail(LUX_ERR_OUT_OF_MEMORY, "scene allocation failed");
    s->device = ctx->device;

    // Instances and the scene-triangle prefix (scene order: instances, then local
    // triangles).
    int64_t total = 0;
    std::vector<int> overrides;
    for (int i = 0; i < d->instance_count; ++i) {
        const lux_instance_desc& in = d->instances[i];
        Instance inst;
        std::memcpy(inst.m, in.object_to_world, sizeof(inst.m));
        bool given = false;
        for (int k = 0; k < 12; ++k) given |= in.world_to_object[k] != 0.0f;
        if (given) std::memcpy(inst.inv, in.world_to_object, sizeof(inst.inv));
        else inverse_affine(inst.m, inst.inv);
        inst.blas = in.mesh;
        inst.first_primitive = static_cast<int>(total);
        s->instances.push_back(inst);
        overrides.push_back(in.material_override);
        total += d->meshes[in.mesh].triangle_count;
        if (total > (int64_t(1) << 30)) {
            delete s;
            return fail(LUX_ERR_INVALID_ARGUMENT, "too many scene triangles (max 2^30)");
        }
    }
    s->triangle_count = static_cast<int>(total);

    // Light-table inputs (scene/scene_prepare.h:268-387): the emissive scene triangles
    // in scene order with their world corners (the device preparation's arithmetic),
    // then the explicit lights; kept so that vertex updates re-derive the tables.  Only
    // emissive triangles are visited: each mesh lists its emissive local triangles once.
    std::vector<float> power_hints(d->material_count, 0.0f);
    for (int i = 0; i < d->material_count; ++i)
        if (is_emissive(d->materials[i])) power_hints[i] = emission_power_hint(d, d->materials[i]);
    std::vector<std::vector<int>> mesh_emissive_tris(d->mesh_count);
    for (int m = 0; m < d->mesh_count; ++m)
        for (int t = 0; t < d->meshes[m].triangle_count; ++t)
            if (is_emissive(d->materials[d->meshes[m].material_ids[t]]))
                mesh_emissive_tris[m].push_back(t);
    s->mesh_emissive.assign(d->mesh_count, 0);
    for (int i = 0; i < d->instance_count; ++i) {
        const lux_mesh_desc& mesh = d->meshes[d->instances[i].mesh];
        const int ov = overrides[i];
        std::vector<int> all;
        const std::vector<int>* local = &mesh_emissive_tris[d->instances[i].mesh];
        if (ov >= 0) {
            if (!is_emissive(d->materials[ov])) continue;
            all.resize(mesh.triangle_count);
            for (int t = 0; t < mesh.triangle_count; ++t) all[t] = t;
            local = &all;
        }
        for (int t : *local) {
            const lux_material& mat = d->materials[ov >= 0 ? ov : mesh.material_ids[t]];
            lux_scene::EmissiveTri e;
            e.triangle = s->instances[i].first_primitive + t;
            e.instance = i;
            e.local = t;
            e.two_sided = mat.emission_two_sided ? 1 : 0;
            for (int k = 0; k < 3; ++k) e.emission[k] = mat.emission[k];
            e.image = mat.emission_source == 1 ? mat.emission_image : -1;
            for (int k = 0; k < 3; ++k) e.image_scale[k] = mat.emission_scale[k];
            e.power_hint = power_hints[ov >= 0 ? ov : mesh.material_ids[t]];
            for (int k = 0; k < 3; ++k) {
                const float* q = mesh.vertices + 3 * size_t(mesh.indices[3 * size_t(t) + k]);
                const V3 w = transform_point(s->instances[i].m, v3(q[0], q[1], q[2]));
                e.w[3 * k] = w.x;
                e.w[3 * k + 1] = w.y;
                e.w[3 * k + 2] = w.z;
            }
            s->emissive.push_back(e);
            s->mesh_emissive[d->instances[i].mesh] = 1;
        }
    }
    // Image lights: texels and running weights (make_image_light_asset,
    // scene/scene_build.h:40-65): weight = max(0, luminance(texel * scale)) * sin(theta)
    // at the row centre, summed in row-major order in float.
    std::vector<float> env_pixels, env_cdf;
    std::vector<pt::EnvLight> env;          // pixels/cdf hold offsets until upload
    std::vector<std::pair<size_t, size_t>> env_offsets;
    for (int i = 0; i < d->light_count; ++i) {
        const lux_light_desc& ld = d->lights[i];
        Light l;
        l.kind = ld.kind;
        l.primitive = -1;
        l.two_sided = 0;
        l.area = 0;
        l.emission = make_f3(ld.value[0], ld.value[1], ld.value[2]);
        V3 vec = v3(ld.vec[0], ld.vec[1], ld.vec[2]);
        if (ld.kind == 2) vec = normalize3(vec);  // add_distant_light stores it normalised
        l.vec = make_f3(vec.x, vec.y, vec.z);
        l.image = -1;
        l.image_scale = make_f3(0, 0, 0);
        float power = std::fmax(1e-6f, luminance(v3(ld.value[0], ld.value[1], ld.value[2])));
        if (ld.kind == 4) {
            const lux_env_image& im = d->images[ld.image];
            const float kPi = 3.14159265358979323846f;
            pt::EnvLight e{};
            e.width = im.width;
            e.height = im.height;
            e.scale = l.emission;
            env_offsets.emplace_back(env_pixels.size(), env_cdf.size());
            float sum = 0;
            for (int y = 0; y < im.height; ++y) {
                float theta = kPi * ((static_cast<float>(y) + 0.5f) / static_cast<float>(im.height));
                float sin_theta = std::fmax(0.0f, std::sin(theta));
                for (int x = 0; x < im.width; ++x) {
                    const float* px = im.pixels + 3 * (static_cast<size_t>(y) * im.width + x);
                    V3 radiance = v3(px[0] * ld.value[0], px[1] * ld.value[1], px[2] * ld.value[2]);
                    sum += std::fmax(0.0f, luminance(radiance)) * sin_theta;
                    env_cdf.push_back(sum);
                    env_pixels.insert(env_pixels.end(), px, px + 3);
                }
            }
            e.total = sum;
            l.primitive = static_cast<int>(env.size());
            env.push_back(e);
            power = std::fmax(1e-6f, sum);
        }
        s->explicit_lights.push_back(l);
        s->explicit_power.push_back(power);
    }
    const LightTables lt = make_light_tables(s->emissive, s->explicit_lights, s->explicit_power,
                                             size_t(total));
    s->area_light_count = lt.area_count;

    // Uploads.
    std::vector<Material> mats;
    for (int i = 0; i < d->material_count; ++i) mats.push_back(to_material(d->materials[i]));
    int st = upload(&s->materials, mats, ctx->stream);
    if (!st) st = upload(&s->d_instances, s->instances, ctx->stream);
    if (!st && !env.empty()) {
        st = upload(&s->env_pixels, env_pixels, ctx->stream);
        if (!st) st = upload(&s->env_cdf, env_cdf, ctx->stream);
        for (size_t k = 0; k < env.size() && !st; ++k) {
            env[k].pixels = s->env_pixels + env_offsets[k].first;
            env[k].cdf = s->env_cdf + env_offsets[k].second;
        }
        if (!st) st = upload(&s->d_env, env, ctx->stream);
    }
    if (!st) st = upload_light_tables(ctx, s, lt);
    // Scene images read by image-emissive materials; the table holds every image (the
    // others with no texels).
    if (!st && d->image_count > 0) {
        std::vector<char> read(d->image_count, 0);
        for (int i = 0; i < d->material_count; ++i)
            if (d->materials[i].emission_source == 1) read[d->materials[i].emission_image] = 1;
        std::vector<float> texels;
        std::vector<size_t> offset(d->image_count, 0);
        std::vector<pt::ImageView> views(d->image_count, pt::ImageView{nullptr, 0, 0});
        for (int i = 0; i < d->image_count; ++i) {
            if (!read[i]) continue;
            const lux_env_image& im = d->images[i];
            offset[i] = texels.size();
            texels.insert(texels.end(), im.pixels, im.pixels + 3 * size_t(im.width) * im.height);
            views[i].width = im.width;
            views[i].height = im.height;
        }
        st = upload(&s->image_pixels, texels, ctx->stream);
        for (int i = 0; i < d->image_count; ++i)
            if (read[i]) views[i].pixels = s->image_pixels + offset[i];
        if (!st) st = upload(&s->d_images, views, ctx->stream);
    }

    // Mesh data to the device, meshes concatenated (the caller's arrays are copied in
    // stream order; pageable sources are staged before each call returns).
    size_t n_vert = 0, n_tri = 0;
    bool any_normals = false, any_uvs = false;
    for (int m = 0; m < d->mesh_count; ++m) {
        n_vert += size_t(d->meshes[m].vertex_count);
        n_tri += size_t(d->meshes[m].triangle_count);
        any_normals |= d->meshes[m].normals != nullptr;
        any_uvs |= d->meshes[m].uvs != nullptr;
    }
    auto dalloc = [&](void** p, size_t bytes) {
        if (st) return;
        if (cudaMalloc(p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            st = fail(LUX_ERR_OUT_OF_MEMORY, "scene allocation failed");
        }
    };
    dalloc(reinterpret_cast<void**>(&s->mesh_data.vertices), sizeof(float) * 3 * n_vert);
    dalloc(reinterpret_cast<void**>(&s->mesh_data.indices), sizeof(uint32_t) * 3 * n_tri);
    dalloc(reinterpret_cast<void**>(&s->mesh_data.material_ids), sizeof(int32_t) * n_tri);
    if (any_normals) dalloc(reinterpret_cast<void**>(&s->mesh_data.normals), sizeof(float) * 3 * n_vert);
    if (any_uvs) dalloc(reinterpret_cast<void**>(&s->mesh_data.uvs), sizeof(float) * 2 * n_vert);
    dalloc(reinterpret_cast<void**>(&s->tri_soup), sizeof(float) * 9 * n_tri);
    dalloc(reinterpret_cast<void**>(&s->tris), sizeof(pt::SceneTri) * size_t(total));
    dalloc(reinterpret_cast<void**>(&s->shading), sizeof(pt::SceneTriShading) * size_t(total));
    std::vector<MeshDev> mesh_dev;
    size_t vo = 0, to = 0;
    auto h2d = [&](void* dst, const void* src, size_t bytes) {
        if (st || !bytes) return;
        cudaError_t err = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
        if (err != cudaSuccess) st = cuda_fail(err, "scene upload");
    };
    for (int m = 0; m < d->mesh_count && !st; ++m) {
        const lux_mesh_desc& mesh = d->meshes[m];
        const size_t nv = size_t(mesh.vertex_count), nt = size_t(mesh.triangle_count);
        h2d(s->mesh_data.vertices + 3 * vo, mesh.vertices, sizeof(float) * 3 * nv);
        h2d(s->mesh_data.indices + 3 * to, mesh.indices, sizeof(uint32_t) * 3 * nt);
        h2d(s->mesh_data.material_ids + to, mesh.material_ids, sizeof(int32_t) * nt);
        if (mesh.normals) h2d(s->mesh_data.normals + 3 * vo, mesh.normals, sizeof(float) * 3 * nv);
        if (mesh.uvs) h2d(s->mesh_data.uvs + 2 * vo, mesh.uvs, sizeof(float) * 2 * nv);
        MeshDev md;
        md.vertices = s->mesh_data.vertices + 3 * vo;
        md.normals = mesh.normals ? s->mesh_data.normals + 3 * vo : nullptr;
        md.uvs = mesh.uvs ? s->mesh_data.uvs + 2 * vo : nullptr;
        md.indices = s->mesh_data.indices + 3 * to;
        md.material_ids = s->mesh_data.material_ids + to;
        md.triangle_count = mesh.triangle_count;
        mesh_dev.push_back(md);
        s->soup_offset.push_back(9 * to);
        s->mesh_vertices.emplace_back(mesh.vertices, mesh.vertices + 3 * nv);
        s->mesh_indices.emplace_back(mesh.indices, mesh.indices + 3 * nt);
        vo += nv;
        to += nt;
    }
    MeshDev* d_meshes = nullptr;
    int* d_overrides = nullptr;
    if (!st) st = upload(&d_meshes, mesh_dev, ctx->stream);
    if (!st) st = upload(&d_overrides, overrides, ctx->stream);

    // World triangles and shading records of every instance, on the device.
    if (!st && total > 0) {
        k_world_triangles<<<prep_blocks(ctx, total), kPrepThreads, 0, ctx->stream>>>(
            d_meshes, s->d_instances, d_overrides, d->instance_count, static_cast<int>(total),
            s->tris, s->shading);
        ctx->launches += 1;
    }

    // BLAS per mesh over its object-space soup (made on the device).
    std::vector<BvhView> views;
    for (int m = 0; m < d->mesh_count && !st; ++m) {
        const MeshDev& md = mesh_dev[m];
        float* soup = s->tri_soup + s->soup_offset[m];
        if (md.triangle_count > 0) {
            k_mesh_soup<<<prep_blocks(ctx, md.triangle_count), kPrepThreads, 0, ctx->stream>>>(
                md.vertices, d->meshes[m].vertex_count, md.indices, md.triangle_count, soup,
                ctx->d_error);
            ctx->launches += 1;
        }
        lux_bvh* b = nullptr;
        st = lux_lbvh_build(ctx, soup, md.triangle_count, LUX_PRIM_TRIANGLES, 30, &b);
        if (!st) {
            s->blas.push_back(b);
            // The path tracer walks each BLAS over its 4-wide nodes.
            st = lbvh_ensure_wide(ctx, b);
        }
        if (!st) views.push_back(b->view());
    }
    if (!st) st = upload(&s->blas_views, views, ctx->stream);

    // TLAS over the instances of non-empty meshes (collect_scene_tlas_build_primitives,
    // scene/scene_prepare.h:441-462): primitive k is instance tlas_instance[k]; boxes
    // from the BLAS roots on the device.
    for (int i = 0; i < d->instance_count; ++i)
        if (d->meshes[d->instances[i].mesh].triangle_count > 0) s->tlas_instance_host.push_back(i);
    const int entries = static_cast<int>(s->tlas_instance_host.size());
    if (!st) st = upload(&s->tlas_instance, s->tlas_instance_host, ctx->stream);
    dalloc(reinterpret_cast<void**>(&s->tlas_boxes), sizeof(float) * 6 * size_t(entries));
    if (!st && entries > 0) {
        k_tlas_boxes<<<(entries + kPrepThreads - 1) / kPrepThreads, kPrepThreads, 0, ctx->stream>>>(
            s->d_instances, s->tlas_instance, s->blas_views, entries, s->tlas_boxes);
        ctx->launches += 1;
    }
    if (!st) st = lux_lbvh_build(ctx, s->tlas_boxes, entries, LUX_PRIM_AABBS, 30, &s->tlas);
    cudaFree(d_meshes);  // waits for the device
    cudaFree(d_overrides);
    if (!st) st = cuda_fail(cudaStreamSynchronize(ctx->stream), "scene upload");
    if (st) {
        scene_free(s);
        delete s;
        return st;
    }

    pt::SceneView& v = s->view;
    v.materials = s->materials;
    v.material_count = d->material_count;
    v.tris = s->tris;
    v.shading = s->shading;
    v.primitive_count = s->triangle_count;
    v.instances = s->d_instances;
    v.instance_count = d->instance_count;
    v.tlas = s->tlas->view();
    v.tlas_instance = s->tlas_instance;
    v.blas = s->blas_views;
    v.env = s->d_env;
    v.images = s->d_images;
    set_light_view(s, lt);
    v.has_two_level = s->tlas->n > 0 && d->instance_count > 0;
    v.has_passthrough = false;
    for (int i = 0; i < d->material_count; ++i)
        v.has_passthrough = v.has_passthrough || d->materials[i].type == pt::kInterface ||
                            d->materials[i].type == pt::kTransparent;
    const lux_camera_desc& c = d->camera;
    v.camera.origin = make_f3(c.origin[0], c.origin[1], c.origin[2]);
    v.camera.lower_left = make_f3(c.lower_left[0], c.lower_left[1], c.lower_left[2]);
    v.camera.horizontal = make_f3(c.horizontal[0], c.horizontal[1], c.horizontal[2]);
    v.camera.vertical = make_f3(c.vertical[0], c.vertical[1], c.vertical[2]);
    v.camera.lens_u = make_f3(c.lens_u[0], c.lens_u[1], c.lens_u[2]);
    v.camera.lens_v = make_f3(c.lens_v[0], c.lens_v[1], c.lens_v[2]);
    v.camera.lens_radius = c.lens_radius;
    *out = s;
    return LUX_OK;
}

// make_perspective_camera (camera/camera.h:77-126) with make_camera_frame (:77-88).
int camera_perspective(const float* origin, const float* look_at, float vfov, float aspect,
                       float lens_radius, float focal_distance, lux_camera_desc* out) {
    const float pi = 3.14159265358979323846f;
    V3 o = v3(origin[0], origin[1], origin[2]);
    V3 at = v3(look_at[0], look_at[1], look_at[2]);
    V3 forward = normalize3(at - o);
    V3 up_world = v3(0, 1, 0);
    V3 right = normalize3(cross3(up_world, forward));
    if (dot3(right, right) == 0) right = normalize3(cross3(v3(0, 0, 1), forward));
    V3 up = cross3(forward, right);
    float theta = vfov * pi / 180.0f;
    float vh = 2.0f * std::tan(theta * 0.5f);
    float vw = aspect * vh;
    float focus = focal_distance > 0 ? focal_distance : len3(at - o);
    if (focus <= 0) focus = 1;
    auto scale = [](V3 v, float s) { return v3(v.x * s, v.y * s, v.z * s); };
    V3 horizontal = scale(right, vw * focus);
    V3 vertical = scale(up, vh * focus);
    V3 f = scale(forward, focus);
    V3 ll = v3(o.x + f.x, o.y + f.y, o.z + f.z);
    V3 h2 = scale(horizontal, 0.5f);
    V3 v2 = scale(vertical, 0.5f);
    ll = v3(ll.x - h2.x, ll.y - h2.y, ll.z - h2.z);
    ll = v3(ll.x - v2.x, ll.y - v2.y, ll.z - v2.z);
    auto put = [](float* d, V3 v) { d[0] = v.x; d[1] = v.y; d[2] = v.z; };
    put(out->origin, o);
    put(out->lower_left, ll);
    put(out->horizontal, horizontal);
    put(out->vertical, vertical);
    put(out->lens_u, right);
    put(out->lens_v, up);
    out->lens_radius = lens_radius;
    return LUX_OK;
}

// ---------------------------------------------------------------- vertex updates
// A vertex update runs on the device in stream order: vertex upload, object-space soup,
// BLAS refit, world positions of every instance of the mesh, instance boxes from the
// refit BLAS's root box (the mesh box: the union of its triangle boxes), TLAS refit.
// The arithmetic is the host restatement's (transform_point, transform_bounds), written
// with round-to-nearest intrinsics so that nothing is contracted, so a refit scene holds
// the values a scene created from the same vertices would.
namespace {

constexpr int kRefitThreads = 256;

__device__ float3 world_point(const float* m, float px, float py, float pz) {
    float x = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], px), __fmul_rn(m[1], py)),
                                  __fmul_rn(m[2], pz)), m[3]);
    float y = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[4], px), __fmul_rn(m[5], py)),
                                  __fmul_rn(m[6], pz)), m[7]);
    float z = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[8], px), __fmul_rn(m[9], py)),
                                  __fmul_rn(m[10], pz)), m[11]);
    float w = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(0.0f, px), __fmul_rn(0.0f, py)),
                                  __fmul_rn(0.0f, pz)), 1.0f);
    if (w == 1.0f) return make_float3(x, y, z);
    return make_float3(__fdiv_rn(x, w), __fdiv_rn(y, w), __fdiv_rn(z, w));
}

// mesh_soup on the device: 9 floats per triangle.
__global__ void k_mesh_soup(const float* vertices, int vertex_count, const uint32_t* indices,
                            int triangle_count, float* soup, int* error) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < triangle_count;
         t += gridDim.x * blockDim.x) {
        for (int k = 0; k < 3; ++k) {
            uint32_t v = indices[3 * size_t(t) + k];
            if (v >= static_cast<uint32_t>(vertex_count)) {  // validated at scene creation
                atomicOr(error, kErrLoopBound);
                v = 0;
            }
            soup[size_t(t) * 9 + 3 * k + 0] = vertices[3 * size_t(v) + 0];
            soup[size_t(t) * 9 + 3 * k + 1] = vertices[3 * size_t(v) + 1];
            soup[size_t(t) * 9 + 3 * k + 2] = vertices[3 * size_t(v) + 2];
        }
    }
}

// World positions of the mesh's triangles in each of its instances (k_world_triangles);
// the .w tags (material, instance, local triangle) are left as uploaded.
__global__ void k_instance_positions(const float* soup, int triangle_count,
                                     const pt::Instance* instances, const int* ids,
                                     int instance_count, pt::SceneTri* tris) {
    int64_t total = int64_t(triangle_count) * instance_count;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total;
         i += int64_t(gridDim.x) * blockDim.x) {
        int j = static_cast<int>(i / triangle_count);
        int t = static_cast<int>(i - int64_t(j) * triangle_count);
        const pt::Instance& inst = instances[ids[j]];
        const float* p = soup + size_t(t) * 9;
        float3 w0 = world_point(inst.m, p[0], p[1], p[2]);
        float3 w1 = world_point(inst.m, p[3], p[4], p[5]);
        float3 w2 = world_point(inst.m, p[6], p[7], p[8]);
        pt::SceneTri* dst = tris + inst.first_primitive + t;
        dst->v0 = make_float4(w0.x, w0.y, w0.z, dst->v0.w);
        dst->v1 = make_float4(w1.x, w1.y, w1.z, dst->v1.w);
        dst->v2 = make_float4(w2.x, w2.y, w2.z, dst->v2.w);
    }
}

// transform_bounds of the mesh box for each TLAS entry of the mesh (instance_box).
__global__ void k_instance_boxes(const float* mesh_box, const pt::Instance* instances,
                                 const int* tlas_instance, const int* entries, int entry_count,
                                 float* tlas_boxes) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= entry_count) return;
    int k = entries[j];
    const pt::Instance& inst = instances[tlas_instance[k]];
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool empty = mesh_box[0] > mesh_box[3] || mesh_box[1] > mesh_box[4] ||
                 mesh_box[2] > mesh_box[5];
    if (!empty) {
        for (int c = 0; c < 8; ++c) {
            int x = c & 1, y = (c >> 1) & 1, z = c >> 2;
            float3 w = world_point(inst.m, x ? mesh_box[3] : mesh_box[0],
                                   y ? mesh_box[4] : mesh_box[1], z ? mesh_box[5] : mesh_box[2]);
            lo[0] = fminf(lo[0], w.x); lo[1] = fminf(lo[1], w.y); lo[2] = fminf(lo[2], w.z);
            hi[0] = fmaxf(hi[0], w.x); hi[1] = fmaxf(hi[1], w.y); hi[2] = fmaxf(hi[2], w.z);
        }
    }
    for (int a = 0; a < 3; ++a) {
        tlas_boxes[6 * k + a] = lo[a];
        tlas_boxes[6 * k + 3 + a] = hi[a];
    }
}

int blocks_for(lux_ctx* ctx, int64_t items) {
    int64_t b = (items + kRefitThreads - 1) / kRefitThreads;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, int64_t(ctx->sm_count) * 8)));
}

// First update of a mesh: device vertex/index buffers and its instance/TLAS-entry lists.
int prepare_refit(lux_scene* s, int mesh) {
    if (s->refit.size() < s->blas.size()) s->refit.resize(s->blas.size());
    lux_scene::MeshRefit& r = s->refit[mesh];
    if (r.vertices) return LUX_OK;
    std::vector<int> lists;
    for (size_t i = 0; i < s->instances.size(); ++i)
        if (s->instances[i].blas == mesh) lists.push_back(static_cast<int>(i));
    int instance_count = static_cast<int>(lists.size());
    for (size_t k = 0; k < s->tlas_instance_host.size(); ++k)
        if (s->instances[s->tlas_instance_host[k]].blas == mesh) lists.push_back(static_cast<int>(k));
    const auto& verts = s->mesh_vertices[mesh];
    const auto& idx = s->mesh_indices[mesh];
    cudaError_t err = cudaMalloc(&r.vertices, sizeof(float) * std::max<size_t>(1, verts.size()));
    if (err == cudaSuccess)
        err = cudaMalloc(&r.indices, sizeof(uint32_t) * std::max<size_t>(1, idx.size()));
    if (err == cudaSuccess)
        err = cudaMalloc(&r.instances, sizeof(int) * std::max<size_t>(1, lists.size()));
    if (err == cudaSuccess && !idx.empty())
        err = cudaMemcpy(r.indices, idx.data(), sizeof(uint32_t) * idx.size(),
                         cudaMemcpyHostToDevice);
    if (err == cudaSuccess && !lists.empty())
        err = cudaMemcpy(r.instances, lists.data(), sizeof(int) * lists.size(),
                         cudaMemcpyHostToDevice);
    if (err != cudaSuccess) {
        cudaFree(r.vertices);
        cudaFree(r.indices);
        cudaFree(r.instances);
        r = lux_scene::MeshRefit{};
        return cuda_fail(err, "mesh update buffers");
    }
    r.instance_count = instance_count;
    r.entry_count = static_cast<int>(lists.size()) - instance_count;
    return LUX_OK;
}

}  // namespace

int scene_update_mesh(lux_ctx* ctx, lux_scene* s, int mesh, const float* vertices, bool sync,
                      bool* view_changed) {
    if (view_changed) *view_changed = false;
    if (mesh < 0 || mesh >= static_cast<int>(s->blas.size()))
        return fail(LUX_ERR_INVALID_ARGUMENT, "mesh out of range");
    if (int st = prepare_refit(s, mesh)) return st;
    std::vector<float>& verts = s->mesh_vertices[mesh];
    std::memcpy(verts.data(), vertices, sizeof(float) * verts.size());
    const lux_scene::MeshRefit& r = s->refit[mesh];
    const int triangle_count = static_cast<int>(s->mesh_indices[mesh].size() / 3);
    const int vertex_count = static_cast<int>(verts.size() / 3);
    if (triangle_count == 0) return LUX_OK;
    float* soup = s->tri_soup + s->soup_offset[mesh];
    cudaStream_t stream = ctx->stream;
    // From pageable memory the copy is staged before the call returns.
    cudaError_t err = cudaMemcpyAsync(r.vertices, verts.data(), sizeof(float) * verts.size(),
                                      cudaMemcpyHostToDevice, stream);
    if (err != cudaSuccess) return cuda_fail(err, "vertex upload");
    k_mesh_soup<<<blocks_for(ctx, triangle_count), kRefitThreads, 0, stream>>>(
        r.vertices, vertex_count, r.indices, triangle_count, soup, ctx->d_error);
    ctx->launches += 1;
    if (int st = lbvh_refit(ctx, s->blas[mesh], soup)) return st;
    // Same node count, so the 4-wide nodes are rebuilt in place (the view is unchanged).
    if (int st = lbvh_ensure_wide(ctx, s->blas[mesh])) return st;
    if (r.instance_count > 0) {
        k_instance_positions<<<blocks_for(ctx, int64_t(triangle_count) * r.instance_count),
                               kRefitThreads, 0, stream>>>(soup, triangle_count, s->d_instances,
                                                           r.instances, r.instance_count, s->tris);
        ctx->launches += 1;
    }
    if (r.entry_count > 0) {
        k_instance_boxes<<<(r.entry_count + kRefitThreads - 1) / kRefitThreads, kRefitThreads, 0,
                           stream>>>(s->blas[mesh]->root, s->d_instances, s->tlas_instance,
                                     r.instances + r.instance_count, r.entry_count, s->tlas_boxes);
        ctx->launches += 1;
        if (int st = lbvh_refit(ctx, s->tlas, s->tlas_boxes)) return st;
    }
    err = cudaGetLastError();
    if (err != cudaSuccess) return cuda_fail(err, "mesh update");
    if (static_cast<size_t>(mesh) < s->mesh_emissive.size() && s->mesh_emissive[mesh]) {
        // The moved emissive triangles' world corners (the arithmetic of
        // k_instance_positions), then every light table.
        const std::vector<uint32_t>& idx = s->mesh_indices[mesh];
        for (lux_scene::EmissiveTri& e : s->emissive) {
            const Instance& inst = s->instances[e.instance];
            if (inst.blas != mesh) continue;
            for (int k = 0; k < 3; ++k) {
                const float* p = verts.data() + 3 * size_t(idx[3 * size_t(e.local) + k]);
                const V3 w = transform_point(inst.m, v3(p[0], p[1], p[2]));
                e.w[3 * k] = w.x;
                e.w[3 * k + 1] = w.y;
                e.w[3 * k + 2] = w.z;
            }
        }
        const LightTables lt = make_light_tables(s->emissive, s->explicit_lights,
                                                 s->explicit_power, size_t(s->triangle_count));
        if (int st = upload_light_tables(ctx, s, lt)) return st;
        set_light_view(s, lt);
        if (view_changed) *view_changed = true;
    }
    if (!sync) return LUX_OK;
    err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) return cuda_fail(err, "mesh update");
    int word = 0;
    err = cudaMemcpy(&word, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return cuda_fail(err, "mesh update");
    if (word) {
        cudaMemset(ctx->d_error, 0, sizeof(int));
        return fail(LUX_ERR_DEVICE_CHECK, "mesh update: device check failed");
    }
    return LUX_OK;
}

}  // namespace lux
