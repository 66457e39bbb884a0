// Host-side scene object of the path tracer (lux_scene) and the wavefront runtime.
#pragma once

#include <cstdint>
#include <vector>

#include "lux_internal.h"
#include "pt_device.cuh"

struct lux_scene {
    int device = 0;
    int triangle_count = 0;
    int area_light_count = 0;
    // Host copies kept for refits and light-table queries.
    std::vector<lux::pt::Instance> instances;
    std::vector<int> mesh_triangle_offset;  // first scene triangle per (instance order)
    std::vector<std::vector<float>> mesh_vertices;     // object space, per mesh
    std::vector<std::vector<uint32_t>> mesh_indices;   // per mesh
    std::vector<int> tlas_instance_host;
    // Device data.
    lux::pt::Material* materials = nullptr;
    lux::pt::SceneTri* tris = nullptr;
    lux::pt::SceneTriShading* shading = nullptr;
    lux::pt::Instance* d_instances = nullptr;
    int* tlas_instance = nullptr;
    lux::BvhView* blas_views = nullptr;
    std::vector<lux_bvh*> blas;
    lux_bvh* tlas = nullptr;
    lux::pt::Light* lights = nullptr;
    lux::pt::AliasEntry* light_alias = nullptr;
    int* primitive_light = nullptr;
    struct MeshData {                   // every mesh's arrays, concatenated (device)
        float* vertices = nullptr;
        float* normals = nullptr;
        float* uvs = nullptr;
        uint32_t* indices = nullptr;
        int32_t* material_ids = nullptr;
    };
    MeshData mesh_data;
    float* tri_soup = nullptr;          // per-mesh object-space soups for refits (device)
    std::vector<size_t> soup_offset;    // float offset of each mesh's soup
    float* tlas_boxes = nullptr;        // instance world boxes (device)
    float* env_pixels = nullptr;        // image-light texels (device)
    float* env_cdf = nullptr;           // image-light running weights (device)
    lux::pt::EnvLight* d_env = nullptr; // image lights (device)
    float* image_pixels = nullptr;      // images read by image-emissive materials (device)
    lux::pt::ImageView* d_images = nullptr;  // every scene image (null pixels if unread)
    // Light tree and the table of the lights outside it (device; null without a tree).
    lux::pt::LightNode* light_tree = nullptr;
    int* light_leaf = nullptr;
    int* light_other_slot = nullptr;
    int* other_lights = nullptr;
    lux::pt::AliasEntry* other_alias = nullptr;
    // Device buffers of vertex updates, allocated on a mesh's first update.
    struct MeshRefit {
        float* vertices = nullptr;       // object space, 3 per vertex
        uint32_t* indices = nullptr;     // 3 per triangle
        int* instances = nullptr;        // instances of the mesh, then their TLAS entries
        int instance_count = 0;
        int entry_count = 0;
    };
    std::vector<MeshRefit> refit;
    // Light-table inputs, kept so that a vertex update re-derives the tables as the
    // reference's re-preparation of a changed scene would.
    struct EmissiveTri {
        int triangle, instance, local;   // scene triangle, its instance and local index
        int two_sided;
        float emission[3];
        int image;                       // image emission: scene image, else -1
        float image_scale[3];
        float power_hint;                // scene_material_emission_power_hint
        float w[9];                      // world positions of the three corners
    };
    std::vector<EmissiveTri> emissive;             // emissive scene triangles, scene order
    std::vector<char> mesh_emissive;               // per mesh: an instance carries emission
    std::vector<lux::pt::Light> explicit_lights;   // point, distant, infinite lights
    std::vector<float> explicit_power;
    struct LightCapacity {                         // element capacity of each light buffer
        size_t lights = 0, alias = 0, primitive = 0, tree = 0, leaf = 0, other_slot = 0,
               other_lights = 0, other_alias = 0;
    };
    LightCapacity light_capacity;
    lux::pt::SceneView view;            // device pointers + counts (TLAS/BLAS filled in)
};

namespace lux {

int scene_create(lux_ctx* ctx, const lux_scene_desc* desc, lux_scene** out);
void scene_free(lux_scene* scene);
// Replaces one mesh's vertices (same count and topology) and refits its BLAS and the TLAS,
// all in stream order on ctx->stream; when an instance of the mesh carries emission, the
// light tables are re-derived on the host and copied in stream order too (the stream is
// waited for only when a table outgrows its buffer).  With sync, waits and reports device
// errors; without, the caller's next synchronisation does.  *view_changed (if given) is
// set when scene->view changed (the light tables were re-derived).
int scene_update_mesh(lux_ctx* ctx, lux_scene* scene, int mesh, const float* vertices,
                      bool sync = true, bool* view_changed = nullptr);
int camera_perspective(const float* origin, const float* look_at, float vfov, float aspect,
                       float lens_radius, float focal_distance, lux_camera_desc* out);

// Wavefront renderer (wavefront.cu).  out is a device pointer: film sums (width*height*3)
// or, when per_sample, every sample's radiance ((pixel*spp + s)*3).  Non-null aov_*
// (device, width*height*3) receive the debug images' per-pixel sums.
// With any debug target (images; path log records, capacity entries, whose counter
// log_count the render zeroes and counts every vertex on), the bounce kernels are the
// debug ones.  walk_counts (device, 3 counters, zeroed by the render) also selects
// them and receives the box tests, triangle tests and instance visits of every walk.
int render(lux_ctx* ctx, const lux_scene* scene, const lux_render_request& req, float* out,
           bool per_sample, float* aov_shadow = nullptr, float* aov_ng = nullptr,
           float* aov_ns = nullptr, lux_path_log_record* log = nullptr,
           unsigned long long* log_count = nullptr, long long log_capacity = 0,
           unsigned long long* walk_counts = nullptr);
int render_ray_counts(lux_ctx* ctx, int64_t* counts);
// Light selection queries (device arrays): sample_scene_light and light_pmf at each
// position, as next-event estimation makes them.
int select_lights(lux_ctx* ctx, const lux_scene* scene, int sampler, const float* positions,
                  const float* select_u, int n, int32_t* light_index, float* pmf,
                  float* eval_pmf);
void render_runtime_free(lux_ctx* ctx);

}  // namespace lux
