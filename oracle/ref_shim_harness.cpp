// Test infrastructure only: calls the drop-in shims (lux_b200/integration/) through the
// reference's OWN types and entry points, as the reference's code would call them once
// the shims replace bvh/gpu_bvh.cu, bvh/bvh_overlap.cu and the wavefront integrator.
// oracle/build.py (build_ref_shim) compiles it with the shims, the reference sources the
// integrator factory needs (integrator/integrator_factory.cpp with LUX_ENABLE_CUDA=1,
// integrator/cpu_path_tracer.cpp, light/light_distribution.cpp,
// scene/prepared_scene_cpu.cpp) and links liblux_gpu.so, into oracle/_ref/libluxshim.so.
// Host code only; nvcc compiles it because the path log record's header includes thrust.
//
// Reference entry points exercised (paths relative to the reference's src/):
//   build_gpu_lbvh, refit_gpu_lbvh, download_bvh_for_validation,
//   validate_gpu_bvh_structure, validate_gpu_bvh_matches_primitives,
//   intersect_gpu_bvh_stackless                    bvh/gpu_bvh.cuh:50-61
//   query_aabb_overlaps_self / _cross             bvh/bvh_overlap.cuh:21-23
//   make_integrator(IntegratorKind::WavefrontPathTracer)->render(...)
//                                                  integrator/integrator_factory.cpp:10-23,
//                                                  integrator/integrator.h:15-22
// Every entry point catches exceptions and returns -1 with the message in `err`.

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "bvh/bvh_overlap.cuh"
#include "bvh/gpu_bvh.cuh"
#include "camera/pinhole_camera.h"
#include "integrator/integrator_factory.h"
#include "integrator/pathstate.cuh"   // PathLogRecord (includes thrust: compiled by nvcc)
#include "integrator/render_context.h"
#include "scene/cornell_box.h"
#include "scene/prepared_scene.h"

#include "ref_scene_desc.h"

#define SHIM_API extern "C" __attribute__((visibility("default")))

namespace {

void copy_error(const char* what, char* err, int errlen) {
    if (!err || errlen <= 0) return;
    std::strncpy(err, what, size_t(errlen) - 1);
    err[errlen - 1] = 0;
}

// Boxes (6 floats each) with their primitive ids as the reference's build input.
std::vector<BvhBuildPrimitive> primitives(const float* boxes, const int* ids, int n) {
    std::vector<BvhBuildPrimitive> out;
    out.reserve(n);
    for (int i = 0; i < n; ++i) {
        const float* b = boxes + size_t(i) * 6;
        AABB box(vec3(b[0], b[1], b[2]), vec3(b[3], b[4], b[5]));
        out.push_back(BvhBuildPrimitive{box, box.centroid(), ids[i], -1, -1, ids[i],
                                        PrimitiveKind::Triangle});
    }
    return out;
}

LightSamplerKind sampler_kind(int light_sampler) {
    return light_sampler == 0 ? LightSamplerKind::Uniform
         : light_sampler == 2 ? LightSamplerKind::Bvh
                              : LightSamplerKind::Power;
}

void copy_film(const Film& film, float* out) {
    if (!out) return;
    for (size_t i = 0; i < film.pixels.size(); ++i) {
        out[3 * i] = film.pixels[i].x;
        out[3 * i + 1] = film.pixels[i].y;
        out[3 * i + 2] = film.pixels[i].z;
    }
}

}  // namespace

SHIM_API void* shim_build(const float* boxes, const int* ids, int n, char* err, int errlen) {
    try {
        return new GpuBvh(build_gpu_lbvh(primitives(boxes, ids, n)));
    } catch (const std::exception& e) {
        copy_error(e.what(), err, errlen);
        return nullptr;
    }
}

SHIM_API void shim_destroy(void* bvh) { delete static_cast<GpuBvh*>(bvh); }

// refit_gpu_lbvh's bool (1 / 0), or -1 on an exception.
SHIM_API int shim_refit(void* bvh, const float* boxes, const int* ids, int n, char* err,
                        int errlen) {
    try {
        return refit_gpu_lbvh(*static_cast<GpuBvh*>(bvh), primitives(boxes, ids, n)) ? 1 : 0;
    } catch (const std::exception& e) {
        copy_error(e.what(), err, errlen);
        return -1;
    }
}

// download_bvh_for_validation: root node, 2n-1 nodes' left / right / first / count and
// boxes, n primitive ids; plus root_bounds (6 floats) of the GpuBvh.
SHIM_API int shim_download(void* bvh, int* root, int* left, int* right, int* first, int* count,
                           float* bounds, int* primitive_ids, float* root_bounds, char* err,
                           int errlen) {
    try {
        const GpuBvh& b = *static_cast<GpuBvh*>(bvh);
        CpuBvhTree tree = download_bvh_for_validation(b);
        *root = tree.root_node;
        for (size_t i = 0; i < tree.nodes.size(); ++i) {
            const CpuBvhNode& nd = tree.nodes[i];
            left[i] = nd.left;
            right[i] = nd.right;
            first[i] = nd.first_primitive;
            count[i] = nd.primitive_count;
            const float box[6] = {nd.bounds.p_min.x, nd.bounds.p_min.y, nd.bounds.p_min.z,
                                  nd.bounds.p_max.x, nd.bounds.p_max.y, nd.bounds.p_max.z};
            std::memcpy(bounds + 6 * i, box, sizeof(box));
        }
        std::copy(tree.primitive_ids.begin(), tree.primitive_ids.end(), primitive_ids);
        const float rb[6] = {b.root_bounds.p_min.x, b.root_bounds.p_min.y, b.root_bounds.p_min.z,
                             b.root_bounds.p_max.x, b.root_bounds.p_max.y, b.root_bounds.p_max.z};
        std::memcpy(root_bounds, rb, sizeof(rb));
        return static_cast<int>(tree.nodes.size());
    } catch (const std::exception& e) {
        copy_error(e.what(), err, errlen);
        return -1;
    }
}

// The two validators; msg receives the second's message when it fails.
SHIM_API int shim_validate(void* bvh, const float* boxes, const int* ids, int n,
                           int* structure_ok, int* matches_ok, char* msg, int msglen) {
    try {
        const GpuBvh& b = *static_cast<GpuBvh*>(bvh);
        std::string m1, m2;
        *structure_ok = validate_gpu_bvh_structure(b, &m1) ? 1 : 0;
        *matches_ok = validate_gpu_bvh_matches_primitives(b, primitives(boxes, ids, n), &m2) ? 1 : 0;
        copy_error((m2.empty() ? m1 : m2).c_str(), msg, msglen);
        return 0;
    } catch (const std::exception& e) {
        copy_error(e.what(), msg, msglen);
        return -1;
    }
}

// intersect_gpu_bvh_stackless: triangles indexed by primitive id (9 floats each), rays in
// the library's 8-float layout.
SHIM_API int shim_intersect(void* bvh, const float* tris, int ntris, const float* rays,
                            int nrays, int* hit_id, float* hit_t, char* err, int errlen) {
    try {
        std::vector<Triangle> t(ntris);
        for (int i = 0; i < ntris; ++i) {
            const float* p = tris + size_t(i) * 9;
            t[i] = Triangle{vec3(p[0], p[1], p[2]), vec3(p[3], p[4], p[5]), vec3(p[6], p[7], p[8])};
        }
        std::vector<Ray> r(nrays);
        for (int i = 0; i < nrays; ++i) {
            const float* p = rays + size_t(i) * 8;
            r[i] = Ray(vec3(p[0], p[1], p[2]), vec3(p[4], p[5], p[6]), p[3], p[7]);
        }
        std::vector<GpuRayHit> hits =
            intersect_gpu_bvh_stackless(*static_cast<GpuBvh*>(bvh), t, r);
        for (int i = 0; i < nrays; ++i) {
            hit_id[i] = hits[i].primitive_id;
            hit_t[i] = hits[i].t;
        }
        return 0;
    } catch (const std::exception& e) {
        copy_error(e.what(), err, errlen);
        return -1;
    }
}

// query_aabb_overlaps_self (right == null) or _cross: pairs (2 ints each, at most
// max_pairs), *truncated; returns found_count, -1 on an exception.
SHIM_API long long shim_overlap(void* left, void* right, int max_pairs, int* pairs,
                                int* truncated, char* err, int errlen) {
    try {
        const GpuBvh& l = *static_cast<GpuBvh*>(left);
        OverlapQueryResult res =
            right ? query_aabb_overlaps_cross(l, *static_cast<GpuBvh*>(right), max_pairs)
                  : query_aabb_overlaps_self(l, max_pairs);
        for (size_t i = 0; i < res.pairs.size(); ++i) {
            pairs[2 * i] = res.pairs[i].a;
            pairs[2 * i + 1] = res.pairs[i].b;
        }
        *truncated = res.truncated ? 1 : 0;
        return res.found_count;
    } catch (const std::exception& e) {
        copy_error(e.what(), err, errlen);
        return -1;
    }
}

// The drop-in render path: the reference's own Scene (from the library's descriptor, or
// the reference's Cornell box when desc is null, with the runner's camera), its
// PreparedScene, make_integrator(WavefrontPathTracer) and Integrator::render with the
// requested debug images and path log, then a second render of the same PreparedScene
// that must give the same film.  Returns the number of path-log records (0 without
// want_log), -1 on an exception.
SHIM_API long long shim_render(const lux_scene_desc* desc, const lux_render_request* req,
                               float* film_out, float* shadow_out, float* ng_out,
                               float* ns_out, int want_log, char* err, int errlen) {
    try {
        Scene scene;
        if (desc) {
            scene = lux_ref_desc::scene_from_desc(*desc);
        } else {
            scene = make_cornell_box();
            scene.camera = make_pinhole_camera(vec3(0, 1, 3.35f), vec3(0, 1, 0.9f), 40.0f,
                                               Float(req->width) / Float(req->height));
        }
        PreparedScene prepared(std::move(scene));
        std::unique_ptr<Integrator> integrator =
            make_integrator(IntegratorKind::WavefrontPathTracer);
        if (integrator->requires_host_bvh()) prepared.prepare_host_bvh();
        if (integrator->requires_gpu_scene()) prepared.prepare_gpu();
        RenderSettings settings;
        settings.max_depth = req->max_depth;
        settings.seed = req->seed;
        settings.frame_index = req->frame_index;
        settings.sample_offset = req->sample_offset;
        settings.light_sampler_kind = sampler_kind(req->light_sampler);
        Film film(req->width, req->height, req->spp);
        Film shadow(req->width, req->height, req->spp), ng = shadow, ns = shadow;
        std::vector<PathLogRecord> log;
        RenderOutputs outputs;
        if (shadow_out) outputs.set(RenderAov::ShadowDebug, &shadow);
        if (ng_out) outputs.set(RenderAov::GeometricNormal, &ng);
        if (ns_out) outputs.set(RenderAov::ShadingNormal, &ns);
        if (want_log) outputs.set_path_log(&log);
        integrator->render(prepared, film, settings, &outputs);
        // A second render of the same prepared scene (the uploaded scene is reused) must
        // give the same film.
        Film again(req->width, req->height, req->spp);
        integrator->render(prepared, again, settings);
        for (size_t i = 0; i < film.pixels.size(); ++i)
            if (film.pixels[i].x != again.pixels[i].x || film.pixels[i].y != again.pixels[i].y ||
                film.pixels[i].z != again.pixels[i].z)
                throw std::runtime_error("second render of the same scene differs");
        copy_film(film, film_out);
        if (shadow_out) copy_film(shadow, shadow_out);
        if (ng_out) copy_film(ng, ng_out);
        if (ns_out) copy_film(ns, ns_out);
        return static_cast<long long>(log.size());
    } catch (const std::exception& e) {
        copy_error(e.what(), err, errlen);
        return -1;
    }
}
