// The reference's wavefront integrator (WavefrontPathTracer, integrator/wavefront_pt.cuh:14-28;
// Integrator::render, integrator/integrator.h:15-22) over liblux_gpu.so.  Replaces
// integrator/wavefront_pt.cu, wavefront_runtime.cu, wavefront_scheduler.cu and
// wavefront_kernels.cu; host code only, compiled by nvcc against the reference's headers
// (integrator/pathstate.cuh, which PathLogRecord lives in, includes thrust).
//
// render() hands the PreparedScene's host scene to the library as a lux_scene_desc
// (materials, meshes, instances, explicit lights, images and camera, field for field
// and in the same order), keeps the uploaded scene while the scene's stamp (identity and
// revision, scene/scene_data.h:152-162) is unchanged, and renders with lux_render /
// lux_render_aovs / lux_render_path_log.  The Film receives the per-pixel sums over its
// samples, as the reference's integrator writes them.  The library prepares the scene on
// the device itself (world triangles, BLAS per mesh, TLAS, light tables), so this
// integrator does not need PreparedScene::prepare_gpu: requires_gpu_scene() is false.

#include <algorithm>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "integrator/pathstate.cuh"
#include "integrator/wavefront_pt.cuh"
#include "scene/scene_data.h"

#include "lux_shim.h"

using lux_shim::check;
using lux_shim::context;

// The integrator's device state: the uploaded scene and the stamp it was made from.
struct WavefrontRuntime {
    lux_scene* scene = nullptr;
    const PreparedScene* prepared = nullptr;
    SceneStamp stamp{};
    ~WavefrontRuntime() {
        if (scene) lux_scene_destroy(scene);
    }
};

namespace {

// The same checks and messages as the reference (integrator/wavefront_pt.cu:12-40).
int checked_image_size(const Film& film) {
    if (film.width <= 0 || film.height <= 0 || film.samples_per_pixel <= 0)
        throw std::runtime_error("WavefrontPathTracer requires a non-empty Film");
    size_t image_size = static_cast<size_t>(film.width) * static_cast<size_t>(film.height);
    if (image_size > static_cast<size_t>(std::numeric_limits<int>::max()))
        throw std::runtime_error("WavefrontPathTracer image is too large");
    if (film.pixels.size() != image_size)
        throw std::runtime_error("WavefrontPathTracer Film pixel storage does not match dimensions");
    return static_cast<int>(image_size);
}

void validate_aov_film(const Film* aov, const Film& beauty, const char* label) {
    if (!aov) return;
    checked_image_size(*aov);
    if (aov->width != beauty.width || aov->height != beauty.height ||
        aov->samples_per_pixel != beauty.samples_per_pixel)
        throw std::runtime_error(std::string("WavefrontPathTracer AOV Film mismatch: ") + label);
}

void put3(float* dst, const vec3& v) {
    dst[0] = v.x;
    dst[1] = v.y;
    dst[2] = v.z;
}

void rows_of(const mat4& m, float* out) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 4; ++j) out[4 * i + j] = m.m[i][j];
}

// The host scene as a lux_scene_desc; `keep` owns the arrays the descriptor points into.
struct SceneArrays {
    std::vector<lux_material> materials;
    std::vector<std::vector<float>> vertices, normals, uvs;
    std::vector<std::vector<uint32_t>> indices;
    std::vector<std::vector<int32_t>> material_ids;
    std::vector<lux_mesh_desc> meshes;
    std::vector<lux_instance_desc> instances;
    std::vector<lux_light_desc> lights;
    std::vector<std::vector<float>> image_pixels;
    std::vector<lux_env_image> images;
    lux_scene_desc desc{};
};

void describe(const Scene& scene, SceneArrays& a) {
    for (const Material& m : scene.materials) {
        lux_material out{};
        out.type = static_cast<int32_t>(m.type);
        put3(out.albedo, m.albedo);
        put3(out.emission, m.emission);
        out.emission_two_sided = m.emission_sidedness == EmissionSidedness::DoubleSided;
        out.roughness = m.roughness;
        out.metallic = m.metallic;
        out.eta = m.eta;
        out.emission_source = m.emission_source == EmissionSourceKind::Image ? 1 : 0;
        out.emission_image = m.emission_image_id;
        put3(out.emission_scale, m.emission_scale);
        a.materials.push_back(out);
    }
    const size_t mesh_count = scene.mesh_assets.size();
    a.vertices.resize(mesh_count);
    a.normals.resize(mesh_count);
    a.uvs.resize(mesh_count);
    a.indices.resize(mesh_count);
    a.material_ids.resize(mesh_count);
    for (size_t k = 0; k < mesh_count; ++k) {
        const SceneMesh& mesh = scene.mesh_assets[k];
        const size_t nv = mesh.vertices.size();
        a.vertices[k].resize(nv * 3);
        a.normals[k].assign(nv * 3, 0.0f);
        a.uvs[k].assign(nv * 2, 0.0f);
        for (size_t v = 0; v < nv; ++v) {
            put3(&a.vertices[k][3 * v], mesh.vertices[v]);
            if (v < mesh.normals.size()) put3(&a.normals[k][3 * v], mesh.normals[v]);
            if (v < mesh.uvs.size()) {
                a.uvs[k][2 * v] = mesh.uvs[v].x;
                a.uvs[k][2 * v + 1] = mesh.uvs[v].y;
            }
        }
        for (const TriangleIndices& t : mesh.indices)
            a.indices[k].insert(a.indices[k].end(), {t.v0, t.v1, t.v2});
        a.material_ids[k].assign(mesh.material_ids.begin(), mesh.material_ids.end());
        lux_mesh_desc d{};
        d.vertices = a.vertices[k].data();
        d.normals = a.normals[k].data();
        d.uvs = a.uvs[k].data();
        d.vertex_count = static_cast<int32_t>(nv);
        d.indices = a.indices[k].data();
        d.material_ids = a.material_ids[k].data();
        d.triangle_count = static_cast<int32_t>(mesh.indices.size());
        a.meshes.push_back(d);
    }
    for (const SceneInstance& inst : scene.instances) {
        lux_instance_desc d{};
        d.mesh = inst.mesh_id;
        d.material_override = inst.material_override;
        rows_of(inst.object_to_world.m, d.object_to_world);
        rows_of(inst.object_to_world.inv, d.world_to_object);
        a.instances.push_back(d);
    }
    for (const Light& l : scene.lights) {
        lux_light_desc d{};
        switch (l.kind) {
            case LightKind::DiffuseArea:   // made from emissive triangles by the library
                continue;
            case LightKind::Point:
                d.kind = 1;
                put3(d.vec, l.point.position);
                put3(d.value, l.point.intensity);
                break;
            case LightKind::Distant:
                d.kind = 2;
                put3(d.vec, l.distant.direction_to_light);
                put3(d.value, l.distant.radiance);
                break;
            case LightKind::UniformInfinite:
                d.kind = 3;
                put3(d.value, l.uniform_infinite.radiance);
                break;
            case LightKind::ImageInfinite:
                d.kind = 4;
                put3(d.value, l.image_infinite.scale);
                d.image = l.image_infinite.image_id;
                break;
        }
        a.lights.push_back(d);
    }
    for (const SceneImageLightAsset& img : scene.image_light_assets) {
        std::vector<float> px(img.pixels.size() * 3);
        for (size_t p = 0; p < img.pixels.size(); ++p) put3(&px[3 * p], img.pixels[p]);
        a.image_pixels.push_back(std::move(px));
    }
    for (size_t k = 0; k < scene.image_light_assets.size(); ++k)
        a.images.push_back(lux_env_image{a.image_pixels[k].data(),
                                         scene.image_light_assets[k].width,
                                         scene.image_light_assets[k].height});
    if (scene.camera.kind != CameraKind::Perspective)
        throw std::runtime_error("WavefrontPathTracer (B200): perspective cameras only");
    const PerspectiveCamera& c = scene.camera.perspective;
    lux_camera_desc cam{};
    put3(cam.origin, c.origin);
    put3(cam.lower_left, c.lower_left);
    put3(cam.horizontal, c.horizontal);
    put3(cam.vertical, c.vertical);
    put3(cam.lens_u, c.lens_u);
    put3(cam.lens_v, c.lens_v);
    cam.lens_radius = c.lens_radius;
    a.desc.materials = a.materials.data();
    a.desc.material_count = static_cast<int32_t>(a.materials.size());
    a.desc.meshes = a.meshes.data();
    a.desc.mesh_count = static_cast<int32_t>(a.meshes.size());
    a.desc.instances = a.instances.data();
    a.desc.instance_count = static_cast<int32_t>(a.instances.size());
    a.desc.lights = a.lights.data();
    a.desc.light_count = static_cast<int32_t>(a.lights.size());
    a.desc.camera = cam;
    a.desc.images = a.images.data();
    a.desc.image_count = static_cast<int32_t>(a.images.size());
}

vec3 v3(const float* f) { return vec3(f[0], f[1], f[2]); }

PathLogRecord from_record(const lux_path_log_record& r) {
    PathLogRecord o;
    o.pixel_index = r.pixel_index;
    o.sample_index = r.sample_index;
    o.depth = r.depth;
    o.triangle_id = r.triangle_id;
    o.primitive_ref = PrimitiveRef{r.instance_id, r.mesh_id, r.local_primitive_id,
                                   static_cast<PrimitiveKind>(r.primitive_kind)};
    o.material_id = r.material_id;
    o.position = v3(r.position);
    o.ng = v3(r.ng);
    o.ns = v3(r.ns);
    o.wo = v3(r.wo);
    o.wi = v3(r.wi);
    o.throughput_before = v3(r.throughput_before);
    o.throughput_after = v3(r.throughput_after);
    o.bsdf_pdf = r.bsdf_pdf;
    o.guide_pdf = r.guide_pdf;
    o.light_pdf = r.light_pdf;
    o.bsdf_pdf_measure = static_cast<PdfMeasure>(r.bsdf_pdf_measure);
    o.guide_pdf_measure = static_cast<PdfMeasure>(r.guide_pdf_measure);
    o.light_pdf_measure = static_cast<PdfMeasure>(r.light_pdf_measure);
    o.sample_source = static_cast<SampleSource>(r.sample_source);
    o.bsdf_flags = r.bsdf_flags;
    o.termination_flags = r.termination_flags;
    o.event_flags = r.event_flags;
    return o;
}

void to_film(const std::vector<float>& sums, Film& film) {
    for (size_t i = 0; i < film.pixels.size(); ++i)
        film.pixels[i] = vec3(sums[3 * i], sums[3 * i + 1], sums[3 * i + 2]);
}

}  // namespace

WavefrontPathTracer::WavefrontPathTracer() : runtime_(std::make_unique<WavefrontRuntime>()) {}

WavefrontPathTracer::~WavefrontPathTracer() = default;

bool WavefrontPathTracer::requires_gpu_scene() const { return false; }

void WavefrontPathTracer::render(const PreparedScene& scene, Film& film,
                                 const RenderSettings& settings, RenderOutputs* outputs) {
    if (settings.max_depth < 0)
        throw std::runtime_error("WavefrontPathTracer requires max_depth >= 0");
    if (settings.batch_size <= 0)
        throw std::runtime_error("WavefrontPathTracer requires batch_size > 0");
    const int image_size = checked_image_size(film);
    Film* shadow = outputs ? outputs->get(RenderAov::ShadowDebug) : nullptr;
    Film* ng = outputs ? outputs->get(RenderAov::GeometricNormal) : nullptr;
    Film* ns = outputs ? outputs->get(RenderAov::ShadingNormal) : nullptr;
    validate_aov_film(shadow, film, "shadow debug");
    validate_aov_film(ng, film, "geometric normal");
    validate_aov_film(ns, film, "shading normal");

    WavefrontRuntime& rt = *runtime_;
    const Scene& host = scene.host_scene();
    const SceneStamp stamp = scene_stamp(host);
    if (!rt.scene || rt.prepared != &scene || rt.stamp.identity != stamp.identity ||
        rt.stamp.revision != stamp.revision) {
        SceneArrays arrays;
        describe(host, arrays);
        lux_scene* uploaded = nullptr;
        check(lux_scene_create(context(), &arrays.desc, &uploaded), "WavefrontPathTracer scene");
        if (rt.scene) lux_scene_destroy(rt.scene);
        rt.scene = uploaded;
        rt.prepared = &scene;
        rt.stamp = stamp;
    }

    lux_render_request req{};
    req.width = film.width;
    req.height = film.height;
    req.spp = film.samples_per_pixel;
    req.max_depth = settings.max_depth;
    req.seed = settings.seed;
    req.frame_index = settings.frame_index;
    req.sample_offset = settings.sample_offset;
    req.light_sampler = static_cast<int32_t>(settings.light_sampler_kind);

    std::vector<float> sums(size_t(image_size) * 3);
    if (outputs && outputs->wants_path_log()) {
        // The reference's bound per render: every path's vertices up to max_depth + 1.
        const long long capacity = static_cast<long long>(image_size) * film.samples_per_pixel *
                                   (settings.max_depth + 1);
        std::vector<lux_path_log_record> records(static_cast<size_t>(capacity));
        int64_t count = 0;
        check(lux_render_path_log(context(), rt.scene, &req, sums.data(), records.data(),
                                  capacity, &count),
              "WavefrontPathTracer path log");
        std::vector<PathLogRecord>& log = *outputs->path_log_records;
        for (int64_t k = 0; k < count; ++k) log.push_back(from_record(records[k]));
    }
    if (shadow || ng || ns) {
        std::vector<float> s(shadow ? sums.size() : 0), g(ng ? sums.size() : 0),
            n(ns ? sums.size() : 0);
        check(lux_render_aovs(context(), rt.scene, &req, sums.data(), shadow ? s.data() : nullptr,
                              ng ? g.data() : nullptr, ns ? n.data() : nullptr),
              "WavefrontPathTracer debug images");
        if (shadow) to_film(s, *shadow);
        if (ng) to_film(g, *ng);
        if (ns) to_film(n, *ns);
    } else if (!(outputs && outputs->wants_path_log())) {
        check(lux_render(context(), rt.scene, &req, sums.data()), "WavefrontPathTracer render");
    }
    to_film(sums, film);
}
