// Test infrastructure only: a C-ABI harness around the reference's OWN GPU wavefront
// path tracer, compiled with nvcc for sm_100a from the reference sources in place
// (oracle/build.py, build_ref_pt_gpu) into oracle/_ref/libluxrefpt.so.  Nothing in the
// product links or loads it: the tests compare this build's images and path logs with
// it, and bench.py times it as the "existing GPU code" bar of the render configurations.
//
// Reference entry points exercised (paths relative to the reference's src/):
//   PreparedScene::prepare_gpu           scene/prepared_scene.h:35-39, prepared_scene.cu
//   WavefrontPathTracer::render          integrator/wavefront_pt.cu:51-84 (the plain
//                                        per-request scheduler,
//                                        integrator/wavefront_scheduler.cu:73-131)
//   RenderOutputs::set_path_log          integrator/render_context.h:65-85, records
//                                        integrator/pathstate.cuh:41-65
//   RenderSettings                       integrator/render_context.h:16-24 (seed set here;
//                                        the reference CLI cannot set it)
//
// The scene comes from the library's own descriptor (oracle/ref_scene_desc.h), so both
// renderers see identical geometry.  Every entry point catches the reference's
// exceptions and returns -1 with the message copied to `err`.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "integrator/pathstate.cuh"
#include "integrator/render_context.h"
#include "integrator/wavefront_pt.cuh"
#include "scene/prepared_scene.h"

#include "ref_scene_desc.h"

#define REFPT_API extern "C" __attribute__((visibility("default")))

namespace {

struct RefPtScene {
    PreparedScene prepared;
    WavefrontPathTracer tracer;
    explicit RefPtScene(Scene scene) : prepared(std::move(scene)) { prepared.prepare_gpu(); }
};

void copy_error(const char* what, char* err, int errlen) {
    if (!err || errlen <= 0) return;
    std::strncpy(err, what, size_t(errlen) - 1);
    err[errlen - 1] = 0;
}

LightSamplerKind sampler_kind(int light_sampler) {
    return light_sampler == 0 ? LightSamplerKind::Uniform
         : light_sampler == 2 ? LightSamplerKind::Bvh
                              : LightSamplerKind::Power;
}

RenderSettings make_settings(const lux_render_request& q, int batch_size) {
    RenderSettings s;
    s.max_depth = q.max_depth;
    s.seed = q.seed;
    s.frame_index = q.frame_index;
    s.sample_offset = q.sample_offset;
    s.light_sampler_kind = sampler_kind(q.light_sampler);
    if (batch_size > 0) s.batch_size = batch_size;
    return s;
}

void copy_film(const Film& film, float* out) {
    if (!out) return;
    for (size_t i = 0; i < film.pixels.size(); ++i) {
        out[3 * i + 0] = film.pixels[i].x;
        out[3 * i + 1] = film.pixels[i].y;
        out[3 * i + 2] = film.pixels[i].z;
    }
}

void to_record(const PathLogRecord& r, lux_path_log_record& o) {
    o.pixel_index = r.pixel_index;
    o.sample_index = r.sample_index;
    o.depth = r.depth;
    o.triangle_id = r.triangle_id;
    o.instance_id = r.primitive_ref.instance_id;
    o.mesh_id = r.primitive_ref.mesh_id;
    o.local_primitive_id = r.primitive_ref.local_primitive_id;
    o.primitive_kind = static_cast<int32_t>(r.primitive_ref.kind);
    o.material_id = r.material_id;
    o.vertex = 0;
    const vec3* v[7] = {&r.position, &r.ng, &r.ns, &r.wo, &r.wi, &r.throughput_before,
                        &r.throughput_after};
    float* d[7] = {o.position, o.ng, o.ns, o.wo, o.wi, o.throughput_before, o.throughput_after};
    for (int k = 0; k < 7; ++k) {
        d[k][0] = v[k]->x;
        d[k][1] = v[k]->y;
        d[k][2] = v[k]->z;
    }
    o.bsdf_pdf = r.bsdf_pdf;
    o.guide_pdf = r.guide_pdf;
    o.light_pdf = r.light_pdf;
    o.bsdf_pdf_measure = static_cast<uint8_t>(r.bsdf_pdf_measure);
    o.guide_pdf_measure = static_cast<uint8_t>(r.guide_pdf_measure);
    o.light_pdf_measure = static_cast<uint8_t>(r.light_pdf_measure);
    o.sample_source = static_cast<uint8_t>(r.sample_source);
    o.bsdf_flags = r.bsdf_flags;
    o.termination_flags = r.termination_flags;
    o.event_flags = r.event_flags;
}

}  // namespace

// Builds the reference's scene from the descriptor and prepares it on the current
// device (its GPU scene and LBVH).  Returns null on failure.
REFPT_API void* refpt_scene_create(const lux_scene_desc* desc, char* err, int errlen) {
    try {
        return new RefPtScene(lux_ref_desc::scene_from_desc(*desc));
    } catch (const std::exception& e) {
        copy_error(e.what(), err, errlen);
        return nullptr;
    }
}

REFPT_API void refpt_scene_destroy(void* scene) { delete static_cast<RefPtScene*>(scene); }

// One WavefrontPathTracer::render of the request (film = the SUM over spp, as the
// reference's Film holds it).  batch_size <= 0 keeps RenderSettings' default (65,536).
// ms receives [0] the render call's duration by CUDA events on the legacy stream, which
// the reference launches on, and [1] its host wall-clock duration (the call returns only
// after its final device-to-host film copy).
REFPT_API int refpt_render(void* scene, const lux_render_request* req, int batch_size,
                           float* film_out, double* ms, char* err, int errlen) {
    try {
        RefPtScene* s = static_cast<RefPtScene*>(scene);
        Film film(req->width, req->height, req->spp);
        RenderSettings settings = make_settings(*req, batch_size);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaDeviceSynchronize();
        auto t0 = std::chrono::steady_clock::now();
        cudaEventRecord(e0, 0);
        s->tracer.render(s->prepared, film, settings);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        auto t1 = std::chrono::steady_clock::now();
        float dev_ms = 0;
        cudaEventElapsedTime(&dev_ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms) {
            ms[0] = dev_ms;
            ms[1] = std::chrono::duration<double, std::milli>(t1 - t0).count();
        }
        copy_film(film, film_out);
        cudaError_t status = cudaGetLastError();
        if (status != cudaSuccess) {
            copy_error(cudaGetErrorString(status), err, errlen);
            return -1;
        }
        return 0;
    } catch (const std::exception& e) {
        copy_error(e.what(), err, errlen);
        return -1;
    }
}

// The same render with the path log on (RenderOutputs::set_path_log).  Records are
// converted to lux_path_log_record and stably sorted by (sample_index, pixel_index):
// within one path the reference appends its vertices in bounce order (one launch per
// bounce), so the stable sort keeps that order and `vertex` numbers it.  *count gets the
// record count; at most capacity records are written (returns 1 if more exist).
REFPT_API int refpt_render_path_log(void* scene, const lux_render_request* req,
                                    int batch_size, float* film_out,
                                    lux_path_log_record* records, int64_t capacity,
                                    int64_t* count, char* err, int errlen) {
    try {
        RefPtScene* s = static_cast<RefPtScene*>(scene);
        Film film(req->width, req->height, req->spp);
        RenderSettings settings = make_settings(*req, batch_size);
        std::vector<PathLogRecord> log;
        RenderOutputs outputs;
        outputs.set_path_log(&log);
        s->tracer.render(s->prepared, film, settings, &outputs);
        copy_film(film, film_out);
        std::vector<size_t> order(log.size());
        std::iota(order.begin(), order.end(), size_t(0));
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
            if (log[a].sample_index != log[b].sample_index)
                return log[a].sample_index < log[b].sample_index;
            return log[a].pixel_index < log[b].pixel_index;
        });
        *count = static_cast<int64_t>(log.size());
        int64_t n = std::min<int64_t>(capacity, static_cast<int64_t>(log.size()));
        int vertex = 0;
        for (int64_t k = 0; k < n; ++k) {
            const PathLogRecord& r = log[order[k]];
            if (k > 0) {
                const PathLogRecord& p = log[order[k - 1]];
                vertex = (p.sample_index == r.sample_index && p.pixel_index == r.pixel_index)
                             ? vertex + 1 : 0;
            }
            to_record(r, records[k]);
            records[k].vertex = vertex;
        }
        return static_cast<int64_t>(log.size()) > capacity ? 1 : 0;
    } catch (const std::exception& e) {
        copy_error(e.what(), err, errlen);
        return -1;
    }
}
