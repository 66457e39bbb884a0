// Test infrastructure only: builds the reference's own `Scene` from the library's
// scene descriptor (lux_scene_desc, include/lux_gpu.h), so that the reference's CPU
// tracer (oracle/ref_harness.cpp) and its GPU wavefront tracer
// (oracle/ref_pt_gpu_harness.cu) render exactly the scene that lux_scene_create
// uploads: the same meshes, instances (with their 3x4 transforms and inverses),
// material overrides, materials, lights, images and camera, in the same order.
//
// Reference calls used (paths relative to the reference's src/):
//   add_scene_mesh / add_scene_instance   scene/scene_edit.h:279-301
//   make_image_light_asset                scene/scene_build.h:41-66
//   add_point_light / add_distant_light / add_uniform_infinite_light
//                                         scene/scene_build.h:9-39
//   ImageInfiniteLight                    light/light.h:79-87 (as
//                                         add_image_infinite_light, scene_build.h:68-89,
//                                         fills it)
//   Camera / PerspectiveCamera            camera/camera.h:29-51
//
// Image lights: a descriptor image referenced by an image light becomes the asset that
// add_image_infinite_light would make with that light's scale; every other image becomes
// an asset with unit scale (an emission image).  Assets keep the descriptor's image
// order, so material emission_image indices carry over unchanged.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <vector>

#include "core/mat4.cuh"
#include "scene/scene_build.h"
#include "scene/scene_data.h"
#include "scene/scene_edit.h"

#include "../include/lux_gpu.h"

namespace lux_ref_desc {

inline mat4 mat_from_rows(const float* r) {
    mat4 m;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 4; ++j) m.m[i][j] = r[4 * i + j];
    return m;
}

inline bool all_zero(const float* r, int n) {
    for (int i = 0; i < n; ++i)
        if (r[i] != 0.0f) return false;
    return true;
}

inline Scene scene_from_desc(const lux_scene_desc& d) {
    Scene scene;
    for (int m = 0; m < d.material_count; ++m) {
        const lux_material& s = d.materials[m];
        Material mat(static_cast<MaterialType>(s.type), vec3(s.albedo[0], s.albedo[1], s.albedo[2]),
                     vec3(s.emission[0], s.emission[1], s.emission[2]), s.roughness, s.metallic,
                     s.eta,
                     s.emission_two_sided ? EmissionSidedness::DoubleSided
                                          : EmissionSidedness::SingleSided);
        if (s.emission_source == 1) {
            mat.emission_source = EmissionSourceKind::Image;
            mat.emission_image_id = s.emission_image;
            mat.emission_scale = vec3(s.emission_scale[0], s.emission_scale[1], s.emission_scale[2]);
        }
        scene.materials.push_back(mat);
    }
    for (int k = 0; k < d.mesh_count; ++k) {
        const lux_mesh_desc& src = d.meshes[k];
        SceneMesh mesh;
        mesh.vertices.reserve(src.vertex_count);
        mesh.normals.reserve(src.vertex_count);
        mesh.uvs.reserve(src.vertex_count);
        for (int v = 0; v < src.vertex_count; ++v) {
            const float* p = src.vertices + 3 * size_t(v);
            mesh.vertices.push_back(vec3(p[0], p[1], p[2]));
            if (src.normals) {
                const float* n = src.normals + 3 * size_t(v);
                mesh.normals.push_back(vec3(n[0], n[1], n[2]));
            } else {
                mesh.normals.push_back(vec3(0));
            }
            if (src.uvs) {
                const float* t = src.uvs + 2 * size_t(v);
                mesh.uvs.push_back(vec2(t[0], t[1]));
            } else {
                mesh.uvs.push_back(vec2(0));
            }
        }
        for (int t = 0; t < src.triangle_count; ++t) {
            const uint32_t* ix = src.indices + 3 * size_t(t);
            mesh.indices.push_back(TriangleIndices{ix[0], ix[1], ix[2]});
            mesh.material_ids.push_back(src.material_ids[t]);
            mesh.boundary_edges.push_back(0);
        }
        add_scene_mesh(scene, std::move(mesh));
    }
    for (int k = 0; k < d.instance_count; ++k) {
        const lux_instance_desc& inst = d.instances[k];
        mat4 m = mat_from_rows(inst.object_to_world);
        Transform xf = all_zero(inst.world_to_object, 12)
                           ? make_transform(m)
                           : Transform(m, mat_from_rows(inst.world_to_object));
        add_scene_instance(scene, inst.mesh, xf, inst.material_override);
    }
    // Image assets in descriptor order (see the header comment for the scale rule).
    for (int k = 0; k < d.image_count; ++k) {
        vec3 scale(1.0f);
        for (int l = 0; l < d.light_count; ++l)
            if (d.lights[l].kind == 4 && d.lights[l].image == k)
                scale = vec3(d.lights[l].value[0], d.lights[l].value[1], d.lights[l].value[2]);
        const lux_env_image& img = d.images[k];
        std::vector<vec3> px(size_t(img.width) * img.height);
        for (size_t p = 0; p < px.size(); ++p)
            px[p] = vec3(img.pixels[3 * p], img.pixels[3 * p + 1], img.pixels[3 * p + 2]);
        scene.image_light_assets.push_back(make_image_light_asset(px, img.width, img.height, scale));
    }
    for (int l = 0; l < d.light_count; ++l) {
        const lux_light_desc& s = d.lights[l];
        vec3 v(s.vec[0], s.vec[1], s.vec[2]);
        vec3 val(s.value[0], s.value[1], s.value[2]);
        if (s.kind == 1) add_point_light(scene, v, val);
        else if (s.kind == 2) add_distant_light(scene, v, val);
        else if (s.kind == 3) add_uniform_infinite_light(scene, val);
        else if (s.kind == 4) {
            if (s.image < 0 || s.image >= static_cast<int>(scene.image_light_assets.size()))
                throw std::runtime_error("scene_from_desc: image light without its image");
            const SceneImageLightAsset& a = scene.image_light_assets[s.image];
            Light light;
            light.kind = LightKind::ImageInfinite;
            light.image_infinite = ImageInfiniteLight{a.pixels.data(), a.cdf.data(), s.image,
                                                      a.width, a.height, a.total_weight, val};
            scene.lights.push_back(light);
            mark_scene_modified(scene);
        } else {
            throw std::runtime_error("scene_from_desc: unknown light kind");
        }
    }
    const lux_camera_desc& c = d.camera;
    scene.camera.kind = CameraKind::Perspective;
    scene.camera.perspective.origin = vec3(c.origin[0], c.origin[1], c.origin[2]);
    scene.camera.perspective.lower_left = vec3(c.lower_left[0], c.lower_left[1], c.lower_left[2]);
    scene.camera.perspective.horizontal = vec3(c.horizontal[0], c.horizontal[1], c.horizontal[2]);
    scene.camera.perspective.vertical = vec3(c.vertical[0], c.vertical[1], c.vertical[2]);
    scene.camera.perspective.lens_u = vec3(c.lens_u[0], c.lens_u[1], c.lens_u[2]);
    scene.camera.perspective.lens_v = vec3(c.lens_v[0], c.lens_v[1], c.lens_v[2]);
    scene.camera.perspective.lens_radius = c.lens_radius;
    return scene;
}

}  // namespace lux_ref_desc
