// Test infrastructure only: a C-ABI harness around the reference's OWN host code,
// compiled from the reference sources in place (see oracle/build.py) into
// oracle/_ref/libluxref.so.  Nothing in the product links or loads this file; the
// tests use it to pin the oracle restatement (oracle/lux_oracle.c) and bench.py
// times it as the reference CPU arm.
//
// Reference entry points exercised (paths relative to the reference's src/):
//   build_cpu_lbvh_tree            bvh/cpu_lbvh_builder.h:163-259
//   lbvh_detail::centroid_to_morton bvh/cpu_lbvh_builder.h:55-61
//   intersect_cpu_bvh_tree         bvh/cpu_bvh_traversal.h:84-95 (CPU stack order)
//   intersect_bvh_device_impl      bvh/bvh_device.cuh:43-90 (GPU stackless order; the
//                                  header is host-compilable because its device
//                                  qualifiers collapse to `inline` outside nvcc)
//   make_cornell_box               scene/cornell_box.h:31-56
//   make_pinhole_camera            camera/pinhole_camera.h:13-17 (camera of
//                                  app/render_runner.cpp:85-90)
//   trace_path                     integrator/cpu_path_tracer.cpp:403-498
//   make_render_sampler            integrator/render_context.h:45-54
//   render_cpu_path_tracer (debug images) integrator/cpu_path_tracer.cpp:160-562
//   path log records (log_path)    integrator/wavefront_kernels.cu:84-138, 356-558 over
//                                  trace_path's walk with the reference's CPU parts
//   load_obj_into_scene_with_result util/obj_loader.cpp:1296-1301
//   make_stanford_bunny_scene, make_lux_cover_scene, make_stanford_dragon_scene
//                                  scene/stanford_bunny.h, scene/lux_cover.h,
//                                  scene/stanford_dragon.h (runner cameras,
//                                  app/render_runner.cpp:148-170)
//
// The stackless node array that intersect_bvh_device_impl walks is produced here
// from the host tree by a plain preorder walk (left child first, escape = the node
// after the subtree), which is the layout bvh/gpu_bvh.cu:241-363 computes on device.

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "bvh/bvh_build_input.h"
#include "bvh/bvh_device.cuh"
#include "bvh/cpu_bvh_traversal.h"
#include "bvh/cpu_lbvh_builder.h"
#include "camera/pinhole_camera.h"
#include "film/pfm.h"
#include "film/ppm.h"
#include "integrator/cpu_path_tracer.h"
#include "integrator/path_transport.cuh"
#include "integrator/render_context.h"
#include "scene/cornell_box.h"
#include "scene/lux_cover.h"
#include "scene/prepared_scene.h"
#include "scene/scene_intersection.h"
#include "scene/scene_light_sampler.h"
#include "scene/stanford_bunny.h"
#include "scene/stanford_dragon.h"
#include "util/obj_loader.h"

// Scenes from the library's own descriptor (lux_scene_desc): meshes, instances,
// materials, lights, images and camera in the order lux_scene_create receives them.
#include "ref_scene_desc.h"

// lux_path_log_record and the LUX_PATH_* flags (the values of PathLogEventFlags and
// PathLogTerminationFlags, integrator/pathstate.cuh:19-39, whose header needs thrust).
#include "../include/lux_gpu.h"

namespace {

std::vector<BvhBuildPrimitive> make_primitives(const float* prims, int n, int kind) {
    std::vector<BvhBuildPrimitive> out;
    out.reserve(n);
    for (int i = 0; i < n; ++i) {
        AABB bounds;
        if (kind == 0) {
            const float* t = prims + size_t(i) * 9;
            Triangle tri{vec3(t[0], t[1], t[2]), vec3(t[3], t[4], t[5]), vec3(t[6], t[7], t[8])};
            bounds = triangle_bounds(tri);
        } else {
            const float* b = prims + size_t(i) * 6;
            bounds = AABB(vec3(b[0], b[1], b[2]), vec3(b[3], b[4], b[5]));
        }
        out.push_back(BvhBuildPrimitive{bounds, bounds.centroid(), i, -1, -1, i,
                                        PrimitiveKind::Triangle});
    }
    return out;
}

std::vector<Triangle> make_triangles(const float* tris, int n) {
    std::vector<Triangle> out(n);
    for (int i = 0; i < n; ++i) {
        const float* t = tris + size_t(i) * 9;
        out[i] = Triangle{vec3(t[0], t[1], t[2]), vec3(t[3], t[4], t[5]), vec3(t[6], t[7], t[8])};
    }
    return out;
}

// Ray record of include/lux_gpu.h: origin.xyz, t_min, direction.xyz, t_max.
Ray make_ray(const float* r) {
    return Ray(vec3(r[0], r[1], r[2]), vec3(r[4], r[5], r[6]), r[3], r[7]);
}

// Preorder (left first) flattening of the host tree into the 32-byte stackless records.
void flatten_preorder(const CpuBvhTree& tree, std::vector<GpuBvhNode>& out) {
    out.assign(tree.nodes.size(), GpuBvhNode{});
    std::vector<int> subtree(tree.nodes.size(), 1);
    // Children always have larger indices in the host layout? Not guaranteed, so
    // compute subtree sizes with an explicit post-order walk.
    std::vector<std::pair<int, int>> stack;  // (node, state)
    stack.push_back({tree.root_node, 0});
    while (!stack.empty()) {
        auto [node, state] = stack.back();
        stack.pop_back();
        const CpuBvhNode& nd = tree.nodes[node];
        if (nd.is_leaf()) { subtree[node] = 1; continue; }
        if (state == 0) {
            stack.push_back({node, 1});
            stack.push_back({nd.right, 0});
            stack.push_back({nd.left, 0});
        } else {
            subtree[node] = 1 + subtree[nd.left] + subtree[nd.right];
        }
    }
    int total = static_cast<int>(tree.nodes.size());
    std::vector<std::pair<int, int>> walk;  // (node, preorder slot)
    walk.push_back({tree.root_node, 0});
    while (!walk.empty()) {
        auto [node, pre] = walk.back();
        walk.pop_back();
        const CpuBvhNode& nd = tree.nodes[node];
        int next = pre + subtree[node];
        GpuBvhNode rec;
        rec.bounds = nd.bounds;
        rec.escape = next < total ? next : -1;
        if (nd.is_leaf()) {
            rec.primitive_id = tree.primitive_ids[nd.first_primitive];
        } else {
            rec.primitive_id = -1;
            walk.push_back({nd.right, pre + 1 + subtree[nd.left]});
            walk.push_back({nd.left, pre + 1});
        }
        out[pre] = rec;
    }
}

template <typename Fn>
void parallel_for(int count, int threads, Fn fn) {
    threads = std::max(1, threads);
    if (threads == 1 || count < 2 * threads) {
        fn(0, count);
        return;
    }
    std::vector<std::thread> pool;
    int chunk = (count + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        int begin = t * chunk;
        int end = std::min(count, begin + chunk);
        if (begin >= end) break;
        pool.emplace_back([=]() { fn(begin, end); });
    }
    for (auto& th : pool) th.join();
}

struct CornellSetup {
    PreparedScene prepared;
    SceneLightSampler lights;
    explicit CornellSetup(int width, int height)
        : prepared(make_scene(width, height)),
          lights(make_scene_light_sampler(prepared.host_scene(), prepared.light_sampling(),
                                          LightSamplerKind::Power)) {
        prepared.prepare_host_bvh();
    }
    static Scene make_scene(int width, int height) {
        Scene scene = make_cornell_box();
        scene.camera = make_pinhole_camera(vec3(0, 1, 3.35f), vec3(0, 1, 0.9f), 40.0f,
                                           Float(width) / Float(height));
        return scene;
    }
};

// One camera sample through the reference loop body of
// integrator/cpu_path_tracer.cpp:525-558 (same draw order: jitter x, jitter y, lens 2D, time).
vec3 reference_sample(const CornellSetup& setup, const RenderSettings& settings,
                      int width, int height, int x, int y, int s) {
    const Scene& scene = setup.prepared.host_scene();
    int pixel = y * width + x;
    SamplerState sampler = make_render_sampler(settings, pixel, s);
    Float jx = sampler_get_1d(sampler);
    Float jy = sampler_get_1d(sampler);
    Float u = (Float(x) + jx) / Float(width);
    Float v = (Float(height - 1 - y) + jy) / Float(height);
    CameraSample cs;
    cs.p_film = vec2(u, v);
    cs.p_lens = sampler_get_2d(sampler);
    cs.time = sampler_get_1d(sampler);
    CameraRay generated = generate_camera_ray(scene.camera, cs);
    if (!generated.valid) return vec3(0);
    return trace_path(scene, setup.prepared.host_bvh(), setup.lights, generated.ray, sampler,
                      settings.max_depth);
}

}  // namespace

extern "C" {

int ref_lbvh_build(const float* prims, int n, int kind, uint32_t* sorted_codes,
                   int32_t* sorted_prim_ids, int32_t* node_left, int32_t* node_right,
                   float* node_bounds) {
    if (n <= 0) return 0;
    std::vector<BvhBuildPrimitive> primitives = make_primitives(prims, n, kind);
    AABB scene_bounds;
    for (const auto& p : primitives) scene_bounds.expand(p.bounds);
    CpuBvhTree tree = build_cpu_lbvh_tree(primitives);
    for (int i = 0; i < n; ++i) {
        int id = tree.primitive_ids[i];
        sorted_prim_ids[i] = id;
        if (sorted_codes) {
            sorted_codes[i] = n == 1 ? 0u
                : lbvh_detail::centroid_to_morton(scene_bounds, primitives[id].centroid);
        }
    }
    int count = static_cast<int>(tree.nodes.size());
    for (int i = 0; i < count; ++i) {
        const CpuBvhNode& nd = tree.nodes[i];
        if (node_left) node_left[i] = nd.is_leaf() ? -1 : nd.left;
        if (node_right) node_right[i] = nd.is_leaf() ? -1 : nd.right;
        if (node_bounds) {
            float* b = node_bounds + size_t(i) * 6;
            b[0] = nd.bounds.p_min.x; b[1] = nd.bounds.p_min.y; b[2] = nd.bounds.p_min.z;
            b[3] = nd.bounds.p_max.x; b[4] = nd.bounds.p_max.y; b[5] = nd.bounds.p_max.z;
        }
    }
    return count;
}

// Builds the host tree over triangles, then traces rays.  mode 0: the reference's GPU
// stackless traversal order (left first) run on the host; mode 1: the reference's CPU
// stack traversal (right child popped first).
int ref_build_and_trace(const float* tris, int ntri, const float* rays, int nrays, int mode,
                        int threads, int32_t* hit_id, float* hit_t) {
    if (ntri <= 0) {
        for (int i = 0; i < nrays; ++i) { hit_id[i] = -1; hit_t[i] = INFINITY; }
        return 0;
    }
    std::vector<BvhBuildPrimitive> primitives = make_primitives(tris, ntri, 0);
    CpuBvhTree tree = build_cpu_lbvh_tree(primitives);
    std::vector<Triangle> triangles = make_triangles(tris, ntri);
    if (mode == 0) {
        std::vector<GpuBvhNode> nodes;
        flatten_preorder(tree, nodes);
        GpuBvhView view{nodes.data(), static_cast<int>(nodes.size()), AABB{}};
        parallel_for(nrays, threads, [&](int begin, int end) {
            for (int i = begin; i < end; ++i) {
                int pid; Float t, u, v;
                bool found = intersect_bvh_device(view, triangles.data(),
                                                  make_ray(rays + size_t(i) * 8), pid, t, u, v);
                hit_id[i] = found ? pid : -1;
                hit_t[i] = found ? t : INFINITY;
            }
        });
    } else {
        parallel_for(nrays, threads, [&](int begin, int end) {
            for (int i = begin; i < end; ++i) {
                int pid; Float t, u, v;
                auto isect = [&](int prim, const Ray& r, CpuBvhPrimitiveHit& h) {
                    Float uu, vv;
                    bool ok = intersect_triangle(r, triangles[prim], h.t, uu, vv);
                    h.u = uu; h.v = vv;
                    return ok;
                };
                bool found = intersect_cpu_bvh_tree(tree, make_ray(rays + size_t(i) * 8), isect,
                                                    pid, t, u, v);
                hit_id[i] = found ? pid : -1;
                hit_t[i] = found ? t : INFINITY;
            }
        });
    }
    return 0;
}

// A built host tree kept alive across calls, so that build and traversal can be timed
// separately (bench.py's reference arm).
struct RefTree {
    CpuBvhTree tree;
    std::vector<Triangle> triangles;
};

void* ref_tree_create(const float* prims, int n, int kind) {
    RefTree* t = new RefTree();
    if (n > 0) {
        t->tree = build_cpu_lbvh_tree(make_primitives(prims, n, kind));
        if (kind == 0) t->triangles = make_triangles(prims, n);
    }
    return t;
}

void ref_tree_destroy(void* handle) { delete static_cast<RefTree*>(handle); }

// Closest hit through intersect_cpu_bvh_tree (the reference CPU traversal).
int ref_tree_trace(void* handle, const float* rays, int nrays, int threads, int32_t* hit_id,
                   float* hit_t) {
    RefTree* t = static_cast<RefTree*>(handle);
    parallel_for(nrays, threads, [&](int begin, int end) {
        for (int i = begin; i < end; ++i) {
            int pid = -1;
            Float tt = INFINITY, u, v;
            bool found = false;
            if (!t->tree.empty()) {
                auto isect = [&](int prim, const Ray& r, CpuBvhPrimitiveHit& h) {
                    Float uu, vv;
                    bool ok = intersect_triangle(r, t->triangles[prim], h.t, uu, vv);
                    h.u = uu; h.v = vv;
                    return ok;
                };
                found = intersect_cpu_bvh_tree(t->tree, make_ray(rays + size_t(i) * 8), isect,
                                               pid, tt, u, v);
            }
            hit_id[i] = found ? pid : -1;
            hit_t[i] = found ? tt : INFINITY;
        }
    });
    return 0;
}

// Cornell box geometry as the reference builds it: 36 triangles (world space, 9
// floats each), their material ids, the 4 materials (type, albedo rgb, emission rgb),
// and the pinhole camera (origin, lower_left, horizontal, vertical).
int ref_cornell_scene(int width, int height, float* tris, int32_t* material_ids,
                      float* materials, float* camera) {
    Scene scene = CornellSetup::make_scene(width, height);
    finalize_scene(scene);
    int count = scene_triangle_count(scene);
    for (int i = 0; i < count; ++i) {
        SceneTriangle st = scene_triangle_view(scene, i);
        const vec3* v = &st.triangle.v0;
        for (int k = 0; k < 3; ++k) {
            tris[i * 9 + k * 3 + 0] = v[k].x;
            tris[i * 9 + k * 3 + 1] = v[k].y;
            tris[i * 9 + k * 3 + 2] = v[k].z;
        }
        material_ids[i] = st.material_id;
    }
    for (size_t m = 0; m < scene.materials.size(); ++m) {
        const Material& mat = scene.materials[m];
        float* o = materials + m * 7;
        o[0] = static_cast<float>(static_cast<int>(mat.type));
        o[1] = mat.albedo.x; o[2] = mat.albedo.y; o[3] = mat.albedo.z;
        o[4] = mat.emission.x; o[5] = mat.emission.y; o[6] = mat.emission.z;
    }
    const PerspectiveCamera& c = scene.camera.perspective;
    const vec3* cv[4] = {&c.origin, &c.lower_left, &c.horizontal, &c.vertical};
    for (int k = 0; k < 4; ++k) {
        camera[k * 3 + 0] = cv[k]->x; camera[k * 3 + 1] = cv[k]->y; camera[k * 3 + 2] = cv[k]->z;
    }
    return count;
}

// Renders pixel rows [y0, y1) of the Cornell box through the reference trace_path with
// settings.seed = seed.  sum/sumsq receive per-pixel RGB sums over samples (row-major,
// full image indexing); samples (optional) receives every sample's RGB as
// [pixel][sample][3] for the rows rendered.
int ref_cornell_render(int width, int height, int spp, int max_depth, uint64_t seed,
                       int y0, int y1, int threads, float* sum, float* sumsq, float* samples) {
    CornellSetup setup(width, height);
    RenderSettings settings;
    settings.max_depth = max_depth;
    settings.seed = seed;
    settings.light_sampler_kind = LightSamplerKind::Power;
    int rows = y1 - y0;
    parallel_for(rows * width, threads, [&](int begin, int end) {
        for (int idx = begin; idx < end; ++idx) {
            int y = y0 + idx / width;
            int x = idx % width;
            int pixel = y * width + x;
            double acc[3] = {0, 0, 0}, acc2[3] = {0, 0, 0};
            for (int s = 0; s < spp; ++s) {
                vec3 L = reference_sample(setup, settings, width, height, x, y, s);
                acc[0] += L.x; acc[1] += L.y; acc[2] += L.z;
                acc2[0] += double(L.x) * L.x; acc2[1] += double(L.y) * L.y;
                acc2[2] += double(L.z) * L.z;
                if (samples) {
                    float* o = samples + (size_t(idx) * spp + s) * 3;
                    o[0] = L.x; o[1] = L.y; o[2] = L.z;
                }
            }
            for (int k = 0; k < 3; ++k) {
                if (sum) sum[size_t(pixel) * 3 + k] = static_cast<float>(acc[k]);
                if (sumsq) sumsq[size_t(pixel) * 3 + k] = static_cast<float>(acc2[k]);
            }
        }
    });
    return 0;
}

// One camera path's surface vertices as the reference's wavefront tracer logs them
// (record_surface_vertex and its call sites in evaluate_hit_kernel,
// integrator/wavefront_kernels.cu:84-138, 356-558), walked the way trace_path walks it
// (integrator/cpu_path_tracer.cpp:403-498) with the reference's own CPU scene query,
// light sampler, direct-light estimate and BSDF sampling.  A miss ends the path
// unlogged.  vertex counts the path's earlier records; sample_index is the sample.
static void log_path(const Scene& scene, const CpuBvh& bvh, const SceneLightSampler& lights,
                     Ray ray, SamplerState& sampler, int max_depth, int pixel, int sample_index,
                     std::vector<lux_path_log_record>& out) {
    vec3 throughput(1);
    PreviousSample previous_sample{0, PdfMeasure::None, SampleSource::Camera, 0, vec3(0)};
    int depth = 0;
    Float eta_scale = 1;
    for (int step = 0; step <= max_depth; ++step) {
        SurfaceHit hit;
        if (!intersect_scene_bvh(scene, bvh, ray, hit)) return;
        const SceneTriangle tri = scene_triangle_view(scene, hit.triangle_id);
        const Material& material = scene.materials[tri.material_id];
        const SurfaceInteraction it =
            make_surface_interaction(hit.position, hit.ng, hit.ns, -ray.direction);
        lux_path_log_record r;
        std::memset(&r, 0, sizeof(r));
        r.pixel_index = pixel;
        r.sample_index = sample_index;
        r.depth = depth;
        r.triangle_id = hit.triangle_id;
        r.instance_id = hit.primitive_ref.instance_id;
        r.mesh_id = hit.primitive_ref.mesh_id;
        r.local_primitive_id = hit.primitive_ref.local_primitive_id;
        r.primitive_kind = static_cast<int32_t>(hit.primitive_ref.kind);
        r.material_id = tri.material_id;
        r.vertex = step;
        auto put = [](float* dst, const vec3& v) { dst[0] = v.x; dst[1] = v.y; dst[2] = v.z; };
        put(r.position, hit.position);
        put(r.ng, it.ng);
        put(r.ns, it.ns);
        put(r.wo, it.wo);
        put(r.throughput_before, throughput);
        r.event_flags = LUX_PATH_EVENT_SURFACE_HIT;
        auto emit = [&](const vec3& after, unsigned termination) {
            put(r.throughput_after, after);
            r.termination_flags = termination;
            if (termination) r.event_flags |= LUX_PATH_EVENT_TERMINATED;
            out.push_back(r);
        };
        const vec3 Le = surface_light_le(lights, hit.triangle_id,
                                         interpolate_triangle_uv(tri, hit.u, hit.v), hit.ng,
                                         -ray.direction);
        if (max_component(Le) > 0 && (emission_uses_unweighted_hit(depth, previous_sample) ||
                                      emission_uses_mis(previous_sample)))
            r.event_flags |= LUX_PATH_EVENT_EMISSION;
        if (is_passthrough_material(material)) {
            r.event_flags |= LUX_PATH_EVENT_PASSTHROUGH | LUX_PATH_EVENT_DELTA;
            put(r.wi, normalize(-it.wo));
            r.bsdf_pdf = 1;
            r.bsdf_pdf_measure = static_cast<uint8_t>(PdfMeasure::Discrete);
            r.sample_source = static_cast<uint8_t>(SampleSource::BSDF);
            r.bsdf_flags = BsdfFlagDeltaTransmission | BsdfFlagTransmission;
            throughput = apply_passthrough(throughput, material);
            if (max_component(throughput) <= 0) return emit(throughput, LUX_PATH_END_ZERO_THROUGHPUT);
            if (step >= max_depth) return emit(throughput, LUX_PATH_END_MAX_DEPTH);
            r.event_flags |= LUX_PATH_EVENT_SPAWNED_RAY;
            emit(throughput, 0);
            ray = spawn_passthrough_ray(hit.position, ray.direction);
            continue;
        }
        if (!material.is_scattering()) return emit(throughput, LUX_PATH_END_NON_SCATTERING);
        if (step >= max_depth || depth >= max_depth)
            return emit(throughput, LUX_PATH_END_MAX_DEPTH);
        if (has_direct_lighting_lobe(material)) {
            LightSampleContext ctx{it.position, it.ng, it.ns};
            Float select_u = sampler_get_1d(sampler);
            Float component_u = sampler_get_1d(sampler);
            vec2 light_u = sampler_get_2d(sampler);
            LightLiSample light = sample_light_li(lights, ctx, select_u, component_u, light_u);
            if (light.valid) {
                r.event_flags |= LUX_PATH_EVENT_DIRECT_LIGHT_SAMPLED;
                DirectLightEstimate direct = estimate_unoccluded_direct_light_li(material, it, light);
                if (direct.pdf_light_solid_angle > 0) {
                    r.light_pdf = direct.pdf_light_solid_angle;
                    r.light_pdf_measure = static_cast<uint8_t>(PdfMeasure::SolidAngle);
                }
                if (direct.valid) r.event_flags |= LUX_PATH_EVENT_DIRECT_LIGHT_VALID;
            }
        }
        BSDFSample sample = sample_bsdf(material, it, sampler_get_2d(sampler));
        put(r.wi, sample.wi);
        r.bsdf_flags = sample.flags;
        r.event_flags |= LUX_PATH_EVENT_BSDF_SAMPLED;
        if (is_delta_bsdf(sample.flags)) r.event_flags |= LUX_PATH_EVENT_DELTA;
        if (sample.pdf > 0) {
            r.bsdf_pdf = sample.pdf;
            r.bsdf_pdf_measure = static_cast<uint8_t>(sample.pdf_measure);
        }
        if (sample.pdf <= 0 || max_component(sample.weight) <= 0)
            return emit(throughput, LUX_PATH_END_INVALID_BSDF);
        vec3 new_throughput = throughput * sample.weight;
        Float new_eta_scale = eta_scale * bsdf_eta_scale_factor(sample);
        r.sample_source = static_cast<uint8_t>(SampleSource::BSDF);
        if (should_apply_russian_roulette(depth)) {
            Float rr_prob = 1;
            if (!survives_russian_roulette(depth, new_throughput, new_eta_scale,
                                           sampler_get_1d(sampler), rr_prob))
                return emit(new_throughput, LUX_PATH_END_RUSSIAN_ROULETTE);
            new_throughput /= rr_prob;
        }
        r.event_flags |= LUX_PATH_EVENT_SPAWNED_RAY;
        emit(new_throughput, 0);
        throughput = new_throughput;
        eta_scale = new_eta_scale;
        previous_sample = PreviousSample{sample.pdf, sample.pdf_measure, SampleSource::BSDF,
                                         sample.flags, hit.position};
        ray = spawn_scatter_ray(hit.position, it.ng, sample.wi);
        ++depth;
    }
}

// A general single-mesh scene through the reference's own authoring and tracing code:
// triangles (world space, 9 floats) with material ids; materials as 11 floats each
// (type, albedo rgb, emission rgb, roughness, metallic, eta, two-sided flag); explicit
// lights as 7 floats (kind 1 point / 2 distant / 3 uniform infinite, vec3, value3);
// camera: origin3, look_at3, vertical fov degrees, aspect (make_pinhole_camera).
// samples receives [pixel][spp][3] for rows [y0, y1).
// mat_ext (optional): 5 floats per material, emission source (1 image), image index and
// emission scale rgb.  uvs (optional): 6 floats per triangle, the corners' texture
// coordinates.  With env_pixels and no image light, the image still becomes scene image 0.
static Scene build_single_mesh_scene(const float* tris, int ntri, const int32_t* mids,
                                     const float* mats, int nmat, const float* lights,
                                     int nlights, const float* cam, const float* env_pixels,
                                     int env_width, int env_height,
                                     const float* mat_ext = nullptr,
                                     const float* uvs = nullptr) {
    Scene scene;
    for (int m = 0; m < nmat; ++m) {
        const float* f = mats + size_t(m) * 11;
        scene.materials.push_back(Material(static_cast<MaterialType>(static_cast<int>(f[0])),
                                           vec3(f[1], f[2], f[3]), vec3(f[4], f[5], f[6]), f[7],
                                           f[8], f[9],
                                           f[10] != 0 ? EmissionSidedness::DoubleSided
                                                      : EmissionSidedness::SingleSided));
        if (mat_ext && mat_ext[5 * m] == 1.0f) {  // Material::image_emissive
            Material& mm = scene.materials.back();
            mm.emission_source = EmissionSourceKind::Image;
            mm.emission_image_id = static_cast<int>(mat_ext[5 * m + 1]);
            mm.emission_scale = vec3(mat_ext[5 * m + 2], mat_ext[5 * m + 3], mat_ext[5 * m + 4]);
        }
    }
    // One append_indexed_mesh (scene/scene_edit.h:98-163) instead of add_triangle per
    // triangle: the same default-mesh data (three vertices per triangle, zero normals and
    // uvs), but one geometry-cache refresh instead of one per triangle, which is
    // quadratic in the triangle count.
    {
        std::vector<vec3> vertices;
        std::vector<vec2> corner_uvs;
        std::vector<TriangleIndices> indices;
        std::vector<int> material_ids(mids, mids + ntri);
        vertices.reserve(size_t(ntri) * 3);
        if (uvs)
            for (int k = 0; k < 3 * ntri; ++k) corner_uvs.push_back(vec2(uvs[2 * k], uvs[2 * k + 1]));
        indices.reserve(ntri);
        for (int t = 0; t < ntri; ++t) {
            const float* v = tris + size_t(t) * 9;
            uint32_t first = static_cast<uint32_t>(vertices.size());
            vertices.push_back(vec3(v[0], v[1], v[2]));
            vertices.push_back(vec3(v[3], v[4], v[5]));
            vertices.push_back(vec3(v[6], v[7], v[8]));
            indices.push_back(TriangleIndices{first, first + 1, first + 2});
        }
        if (ntri > 0) append_indexed_mesh(scene, vertices, {}, corner_uvs, indices, material_ids);
    }
    for (int l = 0; l < nlights; ++l) {
        const float* f = lights + size_t(l) * 7;
        int kind = static_cast<int>(f[0]);
        if (kind == 1) add_point_light(scene, vec3(f[1], f[2], f[3]), vec3(f[4], f[5], f[6]));
        if (kind == 2) add_distant_light(scene, vec3(f[1], f[2], f[3]), vec3(f[4], f[5], f[6]));
        if (kind == 3) add_uniform_infinite_light(scene, vec3(f[4], f[5], f[6]));
        if (kind == 4 && env_pixels) {  // one image: env_pixels, row-major RGB
            std::vector<vec3> px(static_cast<size_t>(env_width) * env_height);
            for (size_t k = 0; k < px.size(); ++k)
                px[k] = vec3(env_pixels[3 * k], env_pixels[3 * k + 1], env_pixels[3 * k + 2]);
            add_image_infinite_light(scene, px, env_width, env_height, vec3(f[4], f[5], f[6]));
        }
    }
    if (env_pixels && scene.image_light_assets.empty()) {
        std::vector<vec3> px(static_cast<size_t>(env_width) * env_height);
        for (size_t k = 0; k < px.size(); ++k)
            px[k] = vec3(env_pixels[3 * k], env_pixels[3 * k + 1], env_pixels[3 * k + 2]);
        scene.image_light_assets.push_back(make_image_light_asset(px, env_width, env_height, vec3(1)));
    }
    scene.camera = make_pinhole_camera(vec3(cam[0], cam[1], cam[2]), vec3(cam[3], cam[4], cam[5]),
                                       cam[6], cam[7]);
    return scene;
}

static LightSamplerKind sampler_kind(int light_sampler) {
    return light_sampler == 0 ? LightSamplerKind::Uniform
         : light_sampler == 2 ? LightSamplerKind::Bvh
                              : LightSamplerKind::Power;
}

int ref_render_scene(const float* tris, int ntri, const int32_t* mids, const float* mats, int nmat,
                     const float* lights, int nlights, const float* cam, int width, int height,
                     int spp, int max_depth, uint64_t seed, int light_sampler, int y0, int y1,
                     int threads, float* samples, const float* env_pixels, int env_width,
                     int env_height, const float* mat_ext, const float* uvs) {
    Scene scene = build_single_mesh_scene(tris, ntri, mids, mats, nmat, lights, nlights, cam,
                                          env_pixels, env_width, env_height, mat_ext, uvs);
    PreparedScene prepared(std::move(scene));
    prepared.prepare_host_bvh();
    SceneLightSampler lights_sampler = make_scene_light_sampler(
        prepared.host_scene(), prepared.light_sampling(),
        sampler_kind(light_sampler));
    RenderSettings settings;
    settings.max_depth = max_depth;
    settings.seed = seed;
    const Scene& sc = prepared.host_scene();
    parallel_for((y1 - y0) * width, threads, [&](int begin, int end) {
        for (int idx = begin; idx < end; ++idx) {
            int y = y0 + idx / width;
            int x = idx % width;
            int pixel = y * width + x;
            for (int s = 0; s < spp; ++s) {
                SamplerState sampler = make_render_sampler(settings, pixel, s);
                Float jx = sampler_get_1d(sampler);
                Float jy = sampler_get_1d(sampler);
                CameraSample cs;
                cs.p_film = vec2((Float(x) + jx) / Float(width),
                                 (Float(height - 1 - y) + jy) / Float(height));
                cs.p_lens = sampler_get_2d(sampler);
                cs.time = sampler_get_1d(sampler);
                CameraRay generated = generate_camera_ray(sc.camera, cs);
                vec3 L = trace_path(sc, prepared.host_bvh(), lights_sampler, generated.ray, sampler,
                                    max_depth);
                float* o = samples + (size_t(idx) * spp + s) * 3;
                o[0] = L.x; o[1] = L.y; o[2] = L.z;
            }
        }
    });
    return 0;
}

// sample_light and light_pmf (scene/scene_light_sampler.h:100-200) of the same scene at
// given shading positions: the picked light index (-1 none), the selection's pmf and
// light_pmf of the picked light.
int ref_select_lights(const float* tris, int ntri, const int32_t* mids, const float* mats,
                      int nmat, const float* lights, int nlights, const float* cam,
                      int light_sampler, const float* positions, const float* select_u, int n,
                      int32_t* light_index, float* pmf, float* eval_pmf) {
    Scene scene = build_single_mesh_scene(tris, ntri, mids, mats, nmat, lights, nlights, cam,
                                          nullptr, 0, 0);
    PreparedScene prepared(std::move(scene));
    SceneLightSampler sampler = make_scene_light_sampler(
        prepared.host_scene(), prepared.light_sampling(), sampler_kind(light_sampler));
    for (int i = 0; i < n; ++i) {
        LightSampleContext ctx{vec3(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]),
                               vec3(0), vec3(0)};
        SampledLight picked = sample_light(sampler, ctx, select_u[i]);
        light_index[i] = picked.light_index;
        pmf[i] = picked.light_index >= 0 ? picked.pmf : 0.0f;
        eval_pmf[i] = picked.light_index >= 0 ? light_pmf(sampler, ctx, picked.light_index) : 0.0f;
    }
    return 0;
}

// render_cpu_path_tracer with its debug images (CpuAovTargets,
// integrator/cpu_path_tracer.cpp:160-397) on a single-mesh scene as ref_render_scene
// builds it (seed = seed): film sums and the shadow / ng / ns images (any may be null),
// width * height * 3 floats each.
int ref_render_aovs(const float* tris, int ntri, const int32_t* mids, const float* mats,
                    int nmat, const float* lights, int nlights, const float* cam, int width,
                    int height, int spp, int max_depth, uint64_t seed, int light_sampler,
                    float* film_out, float* shadow_out, float* ng_out, float* ns_out) {
    Scene scene = build_single_mesh_scene(tris, ntri, mids, mats, nmat, lights, nlights, cam,
                                          nullptr, 0, 0);
    PreparedScene prepared(std::move(scene));
    prepared.prepare_host_bvh();
    RenderSettings settings;
    settings.max_depth = max_depth;
    settings.seed = seed;
    settings.light_sampler_kind = sampler_kind(light_sampler);
    Film film(width, height, spp), shadow(width, height, spp), ng(width, height, spp),
        ns(width, height, spp);
    RenderOutputs outputs;
    outputs.set(RenderAov::ShadowDebug, shadow_out ? &shadow : nullptr);
    outputs.set(RenderAov::GeometricNormal, ng_out ? &ng : nullptr);
    outputs.set(RenderAov::ShadingNormal, ns_out ? &ns : nullptr);
    render_cpu_path_tracer(prepared.host_scene(), prepared.host_bvh(), prepared.light_sampling(),
                           film, settings, &outputs);
    auto copy = [](const Film& f, float* out) {
        if (!out) return;
        for (size_t i = 0; i < f.pixels.size(); ++i) {
            out[3 * i] = f.pixels[i].x;
            out[3 * i + 1] = f.pixels[i].y;
            out[3 * i + 2] = f.pixels[i].z;
        }
    };
    copy(film, film_out);
    copy(shadow, shadow_out);
    copy(ng, ng_out);
    copy(ns, ns_out);
    return 0;
}

// The path log of a render on a single-mesh scene as ref_render_scene builds it
// (seed = seed, sample_offset 0): every path's records in (sample, pixel, vertex) order
// into records (capacity entries); returns the record count, which may exceed capacity
// (then only the first capacity are written).
long long ref_path_log(const float* tris, int ntri, const int32_t* mids, const float* mats,
                       int nmat, const float* lights, int nlights, const float* cam, int width,
                       int height, int spp, int max_depth, uint64_t seed, int light_sampler,
                       lux_path_log_record* records, long long capacity) {
    Scene scene = build_single_mesh_scene(tris, ntri, mids, mats, nmat, lights, nlights, cam,
                                          nullptr, 0, 0);
    PreparedScene prepared(std::move(scene));
    prepared.prepare_host_bvh();
    SceneLightSampler lights_sampler = make_scene_light_sampler(
        prepared.host_scene(), prepared.light_sampling(), sampler_kind(light_sampler));
    RenderSettings settings;
    settings.max_depth = max_depth;
    settings.seed = seed;
    const Scene& sc = prepared.host_scene();
    std::vector<lux_path_log_record> out;
    for (int s = 0; s < spp; ++s) {
        for (int pixel = 0; pixel < width * height; ++pixel) {
            const int x = pixel % width, y = pixel / width;
            SamplerState sampler = make_render_sampler(settings, pixel, s);
            Float jx = sampler_get_1d(sampler);
            Float jy = sampler_get_1d(sampler);
            CameraSample cs;
            cs.p_film = vec2((Float(x) + jx) / Float(width), (Float(height - 1 - y) + jy) / Float(height));
            cs.p_lens = sampler_get_2d(sampler);
            cs.time = sampler_get_1d(sampler);
            CameraRay generated = generate_camera_ray(sc.camera, cs);
            if (!generated.valid) continue;
            log_path(sc, prepared.host_bvh(), lights_sampler, generated.ray, sampler, max_depth,
                     pixel, s, out);
        }
    }
    const long long n = static_cast<long long>(out.size());
    std::memcpy(records, out.data(), sizeof(lux_path_log_record) * size_t(std::min(n, capacity)));
    return n;
}

// ---- OBJ loading and asset scenes

struct RefObj {
    Scene scene;
    ObjLoadResult result;
};

// load_obj_into_scene_with_result into a scene holding 16 placeholder materials (so that
// default and bound material ids up to 15 are valid); counts receives vertex count,
// triangle count and the skipped invalid / non-finite / degenerate triangles.  Returns
// null when the reference's loader fails or loads nothing.
void* ref_obj_load(const char* path, int normal_mode, int reverse, int flip_v, int scale_mode,
                   float target_extent, int center_xz, int ground_to_y, float target_y,
                   const char* const* names, const int32_t* ids, int nbind,
                   int default_material, int32_t* counts) {
    auto* r = new RefObj();
    for (int i = 0; i < 16; ++i) r->scene.materials.push_back(Material::lambert(vec3(0.5f)));
    ObjLoadOptions options;
    options.normal_mode = static_cast<ObjNormalMode>(normal_mode);
    options.reverse_orientation = reverse != 0;
    options.flip_texcoord_v = flip_v != 0;
    options.placement.scale_mode = static_cast<ObjPlacementScaleMode>(scale_mode);
    options.placement.target_extent = target_extent;
    options.placement.center_xz = center_xz != 0;
    options.placement.ground_to_y = ground_to_y != 0;
    options.placement.target_y = target_y;
    options.default_material_id = default_material;
    for (int i = 0; i < nbind; ++i) options.material_bindings[names[i]] = ids[i];
    bool ok = false;
    try {
        ok = load_obj_into_scene_with_result(path, r->scene, options, r->result);
    } catch (const std::exception&) {
        ok = false;
    }
    if (!ok || r->result.mesh_id < 0) {
        delete r;
        return nullptr;
    }
    const SceneMesh& m = r->scene.mesh_assets[r->result.mesh_id];
    counts[0] = static_cast<int32_t>(m.vertices.size());
    counts[1] = static_cast<int32_t>(m.indices.size());
    counts[2] = r->result.skipped_invalid_triangle_count;
    counts[3] = r->result.skipped_nonfinite_triangle_count;
    counts[4] = r->result.skipped_degenerate_triangle_count;
    return r;
}

// The loaded mesh (object space), the instance's object_to_world (row-major 3x4) and
// the mesh box.
int ref_obj_copy(void* handle, float* vertices, float* normals, float* uvs, uint32_t* indices,
                 int32_t* material_ids, float* matrix, float* bounds) {
    auto* r = static_cast<RefObj*>(handle);
    const SceneMesh& m = r->scene.mesh_assets[r->result.mesh_id];
    for (size_t i = 0; i < m.vertices.size(); ++i) {
        vertices[3 * i] = m.vertices[i].x; vertices[3 * i + 1] = m.vertices[i].y;
        vertices[3 * i + 2] = m.vertices[i].z;
        normals[3 * i] = m.normals[i].x; normals[3 * i + 1] = m.normals[i].y;
        normals[3 * i + 2] = m.normals[i].z;
        uvs[2 * i] = m.uvs[i].x; uvs[2 * i + 1] = m.uvs[i].y;
    }
    for (size_t t = 0; t < m.indices.size(); ++t) {
        indices[3 * t] = m.indices[t].v0; indices[3 * t + 1] = m.indices[t].v1;
        indices[3 * t + 2] = m.indices[t].v2;
        material_ids[t] = m.material_ids[t];
    }
    const mat4& x = r->scene.instances[r->result.instance_id].object_to_world.m;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 4; ++j) matrix[4 * i + j] = x.m[i][j];
    bounds[0] = m.bounds.p_min.x; bounds[1] = m.bounds.p_min.y; bounds[2] = m.bounds.p_min.z;
    bounds[3] = m.bounds.p_max.x; bounds[4] = m.bounds.p_max.y; bounds[5] = m.bounds.p_max.z;
    return 0;
}

void ref_obj_free(void* handle) { delete static_cast<RefObj*>(handle); }

// The runner's asset scenes (bunny, dragon, lux-cover) with their cameras.
static bool make_asset_scene(const char* name, const char* root, float aspect, Scene& scene) {
    try {
        std::filesystem::path assets(root);
        std::string n(name);
        if (n == "bunny") {
            scene = make_stanford_bunny_scene(assets);
            scene.camera = make_pinhole_camera(vec3(0.0f, 0.3f, 0.5f), vec3(-0.02f, 0.11f, 0.0f),
                                               40.0f, aspect);
        } else if (n == "dragon") {
            scene = make_stanford_dragon_scene(assets);
            scene.camera = make_pinhole_camera(vec3(0.0f, 0.35f, 0.8f), vec3(0.0f, 0.14f, 0.0f),
                                               42.0f, aspect);
        } else if (n == "lux-cover") {
            scene = make_lux_cover_scene(assets);
            scene.camera = make_pinhole_camera(vec3(0.0f, 0.52f, -3.0f), vec3(0.0f, 0.36f, 0.0f),
                                               32.0f, aspect);
        } else {
            return false;
        }
    } catch (const std::exception&) {
        return false;
    }
    return true;
}

// World triangles (9 floats), material ids and materials (11 floats as ref_render_scene
// takes them) of an asset scene; counts = {triangles, materials}.  With null arrays only
// the counts are written.  Returns -1 when the scene cannot be made.
int ref_asset_scene(const char* name, const char* root, float aspect, int32_t* counts,
                    float* tris, int32_t* material_ids, float* materials) {
    Scene scene;
    if (!make_asset_scene(name, root, aspect, scene)) return -1;
    PreparedScene prepared(std::move(scene));
    const Scene& sc = prepared.host_scene();
    const int count = scene_triangle_count(sc);
    counts[0] = count;
    counts[1] = static_cast<int32_t>(sc.materials.size());
    if (!tris) return 0;
    for (int i = 0; i < count; ++i) {
        SceneTriangle st = scene_triangle_view(sc, i);
        const vec3* v = &st.triangle.v0;
        for (int k = 0; k < 3; ++k) {
            tris[i * 9 + k * 3 + 0] = v[k].x;
            tris[i * 9 + k * 3 + 1] = v[k].y;
            tris[i * 9 + k * 3 + 2] = v[k].z;
        }
        material_ids[i] = st.material_id;
    }
    for (size_t m = 0; m < sc.materials.size(); ++m) {
        const Material& mat = sc.materials[m];
        float* o = materials + m * 11;
        o[0] = static_cast<float>(static_cast<int>(mat.type));
        o[1] = mat.albedo.x; o[2] = mat.albedo.y; o[3] = mat.albedo.z;
        o[4] = mat.emission.x; o[5] = mat.emission.y; o[6] = mat.emission.z;
        o[7] = mat.roughness; o[8] = mat.metallic; o[9] = mat.eta;
        o[10] = mat.emission_sidedness == EmissionSidedness::DoubleSided ? 1.0f : 0.0f;
    }
    return 0;
}

// Rows [y0, y1) of an asset scene through trace_path, as ref_render_scene renders.
int ref_asset_render(const char* name, const char* root, int width, int height, int spp,
                     int max_depth, uint64_t seed, int light_sampler, int y0, int y1,
                     int threads, float* samples) {
    Scene scene;
    if (!make_asset_scene(name, root, Float(width) / Float(height), scene)) return -1;
    PreparedScene prepared(std::move(scene));
    prepared.prepare_host_bvh();
    SceneLightSampler lights_sampler = make_scene_light_sampler(
        prepared.host_scene(), prepared.light_sampling(), sampler_kind(light_sampler));
    RenderSettings settings;
    settings.max_depth = max_depth;
    settings.seed = seed;
    const Scene& sc = prepared.host_scene();
    parallel_for((y1 - y0) * width, threads, [&](int begin, int end) {
        for (int idx = begin; idx < end; ++idx) {
            int y = y0 + idx / width;
            int x = idx % width;
            int pixel = y * width + x;
            for (int s = 0; s < spp; ++s) {
                SamplerState sampler = make_render_sampler(settings, pixel, s);
                Float jx = sampler_get_1d(sampler);
                Float jy = sampler_get_1d(sampler);
                CameraSample cs;
                cs.p_film = vec2((Float(x) + jx) / Float(width),
                                 (Float(height - 1 - y) + jy) / Float(height));
                cs.p_lens = sampler_get_2d(sampler);
                cs.time = sampler_get_1d(sampler);
                CameraRay generated = generate_camera_ray(sc.camera, cs);
                vec3 L = trace_path(sc, prepared.host_bvh(), lights_sampler, generated.ray,
                                    sampler, max_depth);
                float* o = samples + (size_t(idx) * spp + s) * 3;
                o[0] = L.x; o[1] = L.y; o[2] = L.z;
            }
        }
    });
    return 0;
}

// The reference's own image writers on a film of per-pixel sums: kind 0 write_ppm,
// 1 write_debug_ppm_linear, 2 write_pfm (film/ppm.h:37-79, film/pfm.h:27-40).
int ref_write_image(const float* pixels, int width, int height, int spp, const char* path,
                    int kind) {
    std::vector<vec3> px(static_cast<size_t>(width) * height);
    for (size_t i = 0; i < px.size(); ++i)
        px[i] = vec3(pixels[3 * i], pixels[3 * i + 1], pixels[3 * i + 2]);
    if (kind == 0) write_ppm(path, px, width, height, spp);
    else if (kind == 1) write_debug_ppm_linear(path, px, width, height, spp);
    else write_pfm(path, px, width, height, spp);
    return 0;
}

// ---- scenes from lux_scene_desc (any number of meshes and instances, two-level) ----

struct RefDescScene {
    PreparedScene prepared;
    explicit RefDescScene(Scene scene) : prepared(std::move(scene)) {
        prepared.prepare_host_bvh();
    }
};

// The reference's PreparedScene (with its host two-level BVH) of a scene descriptor.
void* ref_desc_scene_create(const lux_scene_desc* desc) {
    return new RefDescScene(lux_ref_desc::scene_from_desc(*desc));
}

void ref_desc_scene_destroy(void* handle) { delete static_cast<RefDescScene*>(handle); }

// trace_path (integrator/cpu_path_tracer.cpp:403-498) for every sample of the pixels
// x in [x0, x1), y in [y0, y1) of the request's frame, with the camera-sample draws of
// render_cpu_path_tracer (cpu_path_tracer.cpp:525-558) and RenderSettings{max_depth,
// seed, frame_index, sample_offset} from the request.  samples (optional) receives
// [pixel of the rectangle, row-major][spp][3]; film (optional) receives the rectangle's
// per-pixel sums in sample order, as the reference's Film accumulates them.
int ref_desc_render(void* handle, const lux_render_request* req, int x0, int y0, int x1,
                    int y1, int threads, float* samples, float* film) {
    const RefDescScene* h = static_cast<const RefDescScene*>(handle);
    const PreparedScene& prepared = h->prepared;
    const Scene& sc = prepared.host_scene();
    SceneLightSampler lights_sampler = make_scene_light_sampler(
        sc, prepared.light_sampling(), sampler_kind(req->light_sampler));
    RenderSettings settings;
    settings.max_depth = req->max_depth;
    settings.seed = req->seed;
    settings.frame_index = req->frame_index;
    settings.sample_offset = req->sample_offset;
    const int width = req->width, height = req->height, spp = req->spp;
    const int cols = x1 - x0;
    parallel_for((y1 - y0) * cols, threads, [&](int begin, int end) {
        for (int idx = begin; idx < end; ++idx) {
            int y = y0 + idx / cols;
            int x = x0 + idx % cols;
            int pixel = y * width + x;
            vec3 sum(0);
            for (int s = 0; s < spp; ++s) {
                SamplerState sampler = make_render_sampler(settings, pixel, s);
                Float jx = sampler_get_1d(sampler);
                Float jy = sampler_get_1d(sampler);
                CameraSample cs;
                cs.p_film = vec2((Float(x) + jx) / Float(width),
                                 (Float(height - 1 - y) + jy) / Float(height));
                cs.p_lens = sampler_get_2d(sampler);
                cs.time = sampler_get_1d(sampler);
                CameraRay generated = generate_camera_ray(sc.camera, cs);
                vec3 L(0);
                if (generated.valid)
                    L = trace_path(sc, prepared.host_bvh(), lights_sampler, generated.ray,
                                   sampler, settings.max_depth);
                sum += L;
                if (samples) {
                    float* o = samples + (size_t(idx) * spp + s) * 3;
                    o[0] = L.x; o[1] = L.y; o[2] = L.z;
                }
            }
            if (film) {
                float* o = film + size_t(idx) * 3;
                o[0] = sum.x; o[1] = sum.y; o[2] = sum.z;
            }
        }
    });
    return 0;
}

}  // extern "C"
