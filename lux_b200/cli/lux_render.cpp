// lux-render: the reference's render command line (app/render_config.h,
// app/render_runner.cpp:294-504) over liblux_gpu.so, for the GPU path (`-gpu`).
//
// Options, defaults, validation, scene names, output paths and messages follow the
// reference: -width/-height/-size, -spp, -depth, -scene, -output (explicit path),
// -out (run directory out/<name>/<stem>.ppm), -gpu, -light-sampler power|uniform|bvh, -time,
// -help.  The render uses RenderSettings' defaults (seed 0, frame 0, sample offset 0),
// so a film equals the reference's `-gpu` film statistically and its CPU film per
// sample.  Images are written as the reference writes them: PPM through write_ppm's
// tone map, PFM when the path ends in ".pfm" (the pixel transforms run on the device,
// lux_film_encode).  This build renders on the GPU only: without -gpu it still renders
// on the GPU and says so.  The asset scenes (bunny, dragon, lux-cover) load their OBJ
// files through lux_obj_load from the reference's asset root (assets/ next to the
// executable, else ./assets).  -debug-aov shadow,ng,ns writes the wavefront tracer's
// debug images (lux_render_aovs) as the reference does; the CPU diagnostics (probes,
// mesh audits, the orientation image) are reported as unsupported.

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <limits>
#include <string>
#include <vector>

#include "lux_gpu.h"

namespace {

using Clock = std::chrono::high_resolution_clock;

struct Config {
    int width = 256;
    int height = 256;
    int spp = 64;
    int max_depth = 4;
    std::string scene = "cornell";
    std::string output;
    int output_mode = 0;  // 0 default run directory, 1 explicit path, 2 run directory
    bool gpu = false;
    bool timing = false;
    bool help = false;
    int light_sampler = 1;  // power
    bool unsupported_option = false;
    std::string unsupported_name;
    // DebugRequest (diagnostics/diagnostic_config.h:51-70).
    int probe_mode = 0;          // 0 none, else camera-hits / path / nee
    bool probe_pixel = false;
    unsigned aov_mask = 0;       // kAov* bits
    int mesh_mode = 0;           // 0 none, else orientation-audit / winding
    std::string debug_output;
};

// DebugAovMask bits and names (diagnostics/diagnostic_config.h).
constexpr unsigned kAovOrientation = 1u, kAovShadow = 2u, kAovNg = 4u, kAovNs = 8u;

bool parse_int(const char* text, int& value, bool allow_zero) {
    char* end = nullptr;
    long v = std::strtol(text, &end, 10);
    if (end == text || *end != '\0') return false;
    if (v < (allow_zero ? 0 : 1) || v > std::numeric_limits<int>::max()) return false;
    value = static_cast<int>(v);
    return true;
}

bool is_opt(const char* a, const char* s, const char* l) {
    return std::strcmp(a, s) == 0 || std::strcmp(a, l) == 0;
}

// parse_debug_aov_list (app/render_config.h:101-137): comma-separated, no empty names.
bool parse_aov_list(const char* text, unsigned& mask) {
    std::string list(text);
    size_t begin = 0;
    for (;;) {
        size_t end = list.find(',', begin);
        std::string name = list.substr(begin, end == std::string::npos ? std::string::npos
                                                                       : end - begin);
        if (name == "orientation") mask |= kAovOrientation;
        else if (name == "shadow") mask |= kAovShadow;
        else if (name == "ng") mask |= kAovNg;
        else if (name == "ns") mask |= kAovNs;
        else return false;
        if (end == std::string::npos) return true;
        begin = end + 1;
    }
}

// parse_render_config (app/render_config.h:196-340).
bool parse(int argc, char** argv, Config& c) {
    bool positional = false;
    for (int i = 1; i < argc; ++i) {
        const char* a = argv[i];
        auto next = [&](const char*& out) {
            if (i + 1 >= argc) return false;
            out = argv[++i];
            return true;
        };
        const char* v = nullptr;
        if (is_opt(a, "-help", "--help")) {
            c.help = true;
        } else if (is_opt(a, "-width", "--width")) {
            if (!next(v) || !parse_int(v, c.width, false)) return false;
        } else if (is_opt(a, "-height", "--height")) {
            if (!next(v) || !parse_int(v, c.height, false)) return false;
        } else if (is_opt(a, "-size", "--size")) {
            if (!next(v) || !parse_int(v, c.width, false)) return false;
            if (!next(v) || !parse_int(v, c.height, false)) return false;
        } else if (is_opt(a, "-spp", "--spp")) {
            if (!next(v) || !parse_int(v, c.spp, false)) return false;
        } else if (is_opt(a, "-depth", "--depth")) {
            if (!next(v) || !parse_int(v, c.max_depth, true)) return false;
        } else if (is_opt(a, "-scene", "--scene")) {
            if (!next(v)) return false;
            c.scene = v;
        } else if (is_opt(a, "-output", "--output")) {
            if (!next(v)) return false;
            c.output = v;
            c.output_mode = 1;
        } else if (is_opt(a, "-out", "--out")) {
            if (!next(v)) return false;
            c.output = v;
            c.output_mode = 2;
        } else if (is_opt(a, "-gpu", "--gpu")) {
            c.gpu = true;
        } else if (is_opt(a, "-light-sampler", "--light-sampler")) {
            if (!next(v)) return false;
            if (std::strcmp(v, "power") == 0) {
                c.light_sampler = 1;
            } else if (std::strcmp(v, "uniform") == 0) {
                c.light_sampler = 0;
            } else if (std::strcmp(v, "bvh") == 0) {
                c.light_sampler = 2;
            } else {
                return false;
            }
        } else if (is_opt(a, "-time", "--time")) {
            c.timing = true;
        } else if (is_opt(a, "-debug-probe", "--debug-probe")) {
            int px = 0, py = 0;
            if (!next(v) || !parse_int(v, px, true)) return false;
            if (!next(v) || !parse_int(v, py, true)) return false;
            c.probe_pixel = true;
            if (c.probe_mode == 0) c.probe_mode = 1;
        } else if (is_opt(a, "-debug-mode", "--debug-mode")) {
            if (!next(v)) return false;
            if (std::strcmp(v, "camera-hits") == 0) c.probe_mode = 1;
            else if (std::strcmp(v, "path") == 0) c.probe_mode = 2;
            else if (std::strcmp(v, "nee") == 0) c.probe_mode = 3;
            else return false;
        } else if (is_opt(a, "-debug-aov", "--debug-aov")) {
            if (!next(v) || !parse_aov_list(v, c.aov_mask)) return false;
        } else if (is_opt(a, "-debug-output", "--debug-output")) {
            if (!next(v)) return false;
            c.debug_output = v;
        } else if (is_opt(a, "-debug-samples", "--debug-samples") ||
                   is_opt(a, "-debug-max-hits", "--debug-max-hits")) {
            int n = 0;
            if (!next(v) || !parse_int(v, n, false)) return false;
        } else if (is_opt(a, "-debug-mesh", "--debug-mesh")) {
            if (!next(v)) return false;
            if (std::strcmp(v, "orientation-audit") == 0) c.mesh_mode = 1;
            else if (std::strcmp(v, "winding") == 0) c.mesh_mode = 2;
            else return false;
        } else if (is_opt(a, "-debug-triangle", "--debug-triangle")) {
            int t = 0;
            if (!next(v) || !parse_int(v, t, true)) return false;
            if (c.mesh_mode == 0) c.mesh_mode = 2;
        } else if (a[0] == '-') {
            return false;
        } else {
            // The one positional argument is the output path, alone on the command line.
            if (positional || argc != 2) return false;
            positional = true;
            c.output = a;
            c.output_mode = 1;
        }
    }
    // validate_debug_request (app/render_config.h:167-175): one debug category at most;
    // a probe needs its pixel.
    const int categories = (c.probe_mode ? 1 : 0) + (c.mesh_mode ? 1 : 0) + (c.aov_mask ? 1 : 0);
    if (categories > 1 || (c.probe_mode && !c.probe_pixel)) return false;
    // The probes, mesh diagnostics and the orientation image are CPU diagnostics.
    if (c.probe_mode || c.mesh_mode || (c.aov_mask & kAovOrientation)) {
        c.unsupported_option = true;
        c.unsupported_name = c.probe_mode ? "-debug-probe" : c.mesh_mode ? "-debug-mesh"
                                                                        : "-debug-aov orientation";
    }
    return true;
}

// debug_aov_output_path (diagnostics/diagnostic_config.h:32-43): the image's name before
// the prefix's .ppm / .pfm extension.
std::string aov_path(const std::string& prefix, const char* name) {
    std::string base = prefix, ext = ".ppm";
    if (base.size() >= 4) {
        std::string suffix = base.substr(base.size() - 4);
        if (suffix == ".ppm" || suffix == ".pfm") {
            ext = suffix;
            base.resize(base.size() - 4);
        }
    }
    return base + "_" + name + ext;
}

void usage(const char* exe) {
    std::printf(
        "Usage: %s [scene] [options]\n"
        "  -scene NAME             cornell, direct-light, point-light, distant-light,\n"
        "                          uniform-env, image-env, transparent-filter, bunny,\n"
        "                          dragon, lux-cover\n"
        "  -width N / -height N / -size W H   film size (default 256x256)\n"
        "  -spp N                  samples per pixel (default 64)\n"
        "  -depth N                maximum path depth (default 4)\n"
        "  -light-sampler KIND     power (default), uniform or bvh\n"
        "  -output PATH            image path (.ppm, or .pfm for linear floats)\n"
        "  -out NAME               write out/NAME/<NAME>.ppm\n"
        "  -gpu                    render with the GPU path (the only path of this build)\n"
        "  -time                   print a timing breakdown\n"
        "  -debug-aov LIST         debug images: shadow, ng, ns (comma-separated)\n"
        "  -debug-output PATH      prefix of the debug images (default: the image path)\n",
        exe);
}

// ---------------------------------------------------------------- scenes
struct SceneData {
    std::vector<lux_material> materials;
    std::vector<float> vertices;         // default mesh, 3 vertices per triangle
    std::vector<uint32_t> indices;
    std::vector<int32_t> material_ids;
    std::vector<lux_light_desc> lights;
    std::vector<std::vector<float>> image_pixels;
    std::vector<lux_env_image> images;
    float cam_origin[3], cam_look_at[3], cam_vfov;
    std::vector<lux_obj_mesh*> obj_meshes;  // extra meshes, one instance each
    ~SceneData() {
        for (lux_obj_mesh* m : obj_meshes) lux_obj_mesh_free(m);
    }
};

lux_material mat(int type, float r, float g, float b, float er = 0, float eg = 0, float eb = 0,
                 float roughness = 0.5f, float metallic = 0.0f, float eta = 1.5f) {
    lux_material m{};
    m.type = type;
    m.albedo[0] = r; m.albedo[1] = g; m.albedo[2] = b;
    m.emission[0] = er; m.emission[1] = eg; m.emission[2] = eb;
    m.emission_two_sided = 0;
    m.roughness = roughness; m.metallic = metallic; m.eta = eta;
    return m;
}
constexpr int kLambert = 0, kThinLambert = 1, kGgx = 2, kDielectric = 3, kInterface = 4,
              kTransparent = 5;
int add_material(SceneData& s, const lux_material& m) {
    s.materials.push_back(m);
    return static_cast<int>(s.materials.size()) - 1;
}
// Material::lambert / emissive / tinted_filter / interface (material/material.h:43-103).
int lambert(SceneData& s, float r, float g, float b) { return add_material(s, mat(kLambert, r, g, b)); }
int emissive(SceneData& s, float r, float g, float b) { return add_material(s, mat(kLambert, 0, 0, 0, r, g, b)); }
int tinted(SceneData& s, float r, float g, float b) { return add_material(s, mat(kTransparent, r, g, b)); }
int interface_mat(SceneData& s) { return add_material(s, mat(kInterface, 1, 1, 1)); }

struct V { float x, y, z; };
// add_triangle / add_quad (scene/scene_edit.h:66-96, 261-265): loose triangles in the
// default mesh, quad (p0, p1, p2, p3) as (p0, p1, p2), (p0, p2, p3).
void triangle(SceneData& s, V a, V b, V c, int material) {
    uint32_t first = static_cast<uint32_t>(s.vertices.size() / 3);
    for (V p : {a, b, c}) s.vertices.insert(s.vertices.end(), {p.x, p.y, p.z});
    s.indices.insert(s.indices.end(), {first, first + 1, first + 2});
    s.material_ids.push_back(material);
}
void quad(SceneData& s, V p0, V p1, V p2, V p3, int material) {
    triangle(s, p0, p1, p2, material);
    triangle(s, p0, p2, p3, material);
}
void camera(SceneData& s, V o, V at, float vfov) {
    s.cam_origin[0] = o.x; s.cam_origin[1] = o.y; s.cam_origin[2] = o.z;
    s.cam_look_at[0] = at.x; s.cam_look_at[1] = at.y; s.cam_look_at[2] = at.z;
    s.cam_vfov = vfov;
}

// make_cornell_box (scene/cornell_box.h:31-56) with the runner's camera
// (app/render_runner.cpp:85-90).
void cornell(SceneData& s) {
    int white = lambert(s, 0.78f, 0.78f, 0.74f);
    int red = lambert(s, 0.65f, 0.05f, 0.05f);
    int green = lambert(s, 0.12f, 0.45f, 0.15f);
    int light = emissive(s, 15.0f, 14.0f, 12.0f);
    quad(s, {-1, 0, 2}, {1, 0, 2}, {1, 0, 0}, {-1, 0, 0}, white);
    quad(s, {-1, 2, 0}, {1, 2, 0}, {1, 2, 2}, {-1, 2, 2}, white);
    quad(s, {-1, 0, 0}, {1, 0, 0}, {1, 2, 0}, {-1, 2, 0}, white);
    quad(s, {-1, 0, 2}, {-1, 0, 0}, {-1, 2, 0}, {-1, 2, 2}, red);
    quad(s, {1, 0, 0}, {1, 0, 2}, {1, 2, 2}, {1, 2, 0}, green);
    auto box = [&](V lo, V hi, int m) {  // cornell_box_detail::add_box (:10-27)
        V p000{lo.x, lo.y, lo.z}, p100{hi.x, lo.y, lo.z}, p110{hi.x, hi.y, lo.z},
            p010{lo.x, hi.y, lo.z}, p001{lo.x, lo.y, hi.z}, p101{hi.x, lo.y, hi.z},
            p111{hi.x, hi.y, hi.z}, p011{lo.x, hi.y, hi.z};
        quad(s, p000, p100, p110, p010, m);
        quad(s, p101, p001, p011, p111, m);
        quad(s, p001, p000, p010, p011, m);
        quad(s, p100, p101, p111, p110, m);
        quad(s, p010, p110, p111, p011, m);
        quad(s, p001, p101, p100, p000, m);
    };
    box({-0.65f, 0, 0.35f}, {-0.15f, 0.8f, 0.9f}, white);
    box({0.25f, 0, 0.75f}, {0.75f, 1.2f, 1.35f}, white);
    quad(s, {-0.35f, 1.99f, 0.75f}, {0.35f, 1.99f, 0.75f}, {0.35f, 1.99f, 1.35f},
         {-0.35f, 1.99f, 1.35f}, light);
    camera(s, {0, 1, 3.35f}, {0, 1, 0.9f}, 40.0f);
}

// make_direct_light_test_scene (scene/direct_light_test.h:9-24), runner camera :92-96.
void direct_light(SceneData& s) {
    int receiver = lambert(s, 0.8f, 0.8f, 0.8f);
    int light = emissive(s, 1.0f, 1.0f, 1.0f);
    quad(s, {-1, 0, 1}, {1, 0, 1}, {1, 0, -1}, {-1, 0, -1}, receiver);
    quad(s, {-0.2f, 1.4f, -0.2f}, {0.2f, 1.4f, -0.2f}, {0.2f, 1.4f, 0.2f}, {-0.2f, 1.4f, 0.2f},
         light);
    camera(s, {0, 1.2f, 3.0f}, {0, 0, 0}, 35.0f);
}

// make_probe_base_scene (app/render_runner.cpp:98-109) and its light variants.
void probe_base(SceneData& s) {
    int receiver = lambert(s, 0.75f, 0.75f, 0.75f);
    quad(s, {-1.2f, 0, 1.2f}, {1.2f, 0, 1.2f}, {1.2f, 0, -1.2f}, {-1.2f, 0, -1.2f}, receiver);
    camera(s, {0, 0.8f, 2.8f}, {0, 0, 0}, 35.0f);
}
void add_light(SceneData& s, int kind, V vec, V value) {
    lux_light_desc l{};
    l.kind = kind;
    l.vec[0] = vec.x; l.vec[1] = vec.y; l.vec[2] = vec.z;
    l.value[0] = value.x; l.value[1] = value.y; l.value[2] = value.z;
    s.lights.push_back(l);
}
void point_light(SceneData& s) {
    probe_base(s);
    add_light(s, 1, {0.0f, 1.6f, 0.2f}, {25.0f, 25.0f, 25.0f});
}
void distant_light(SceneData& s) {
    probe_base(s);
    // normalize(vec3(-0.4, 1.0, 0.3)) (core/vec3.cuh:62-66: v * (1 / length)).
    float x = -0.4f, y = 1.0f, z = 0.3f;
    float inv = 1.0f / std::sqrt(x * x + y * y + z * z);
    add_light(s, 2, {x * inv, y * inv, z * inv}, {1.2f, 1.2f, 1.2f});
}
void uniform_env(SceneData& s) {
    probe_base(s);
    add_light(s, 3, {0, 0, 0}, {0.15f, 0.18f, 0.25f});
}
// make_image_env_scene (app/render_runner.cpp:127-136): a 2x2 latitude-longitude image.
void image_env(SceneData& s) {
    probe_base(s);
    s.image_pixels.push_back({1.4f, 1.0f, 0.7f, 0.2f, 0.3f, 0.8f,
                              0.1f, 0.2f, 0.5f, 0.8f, 1.1f, 1.5f});
    lux_env_image im{};
    im.width = 2;
    im.height = 2;
    s.images.push_back(im);
    add_light(s, 4, {0, 0, 0}, {0.35f, 0.35f, 0.35f});
    s.lights.back().image = 0;
}
// make_transparent_filter_scene (scene/transparent_filter.h:9-40), runner camera :138-144.
void transparent_filter(SceneData& s) {
    int receiver = lambert(s, 0.75f, 0.75f, 0.75f);
    int area_light = emissive(s, 8.0f, 8.0f, 8.0f);
    int filter = tinted(s, 0.25f, 0.65f, 1.0f);
    int clear = interface_mat(s);
    int card = emissive(s, 3.0f, 2.2f, 1.2f);
    quad(s, {-1.6f, 0, 1.5f}, {1.6f, 0, 1.5f}, {1.6f, 0, -1.5f}, {-1.6f, 0, -1.5f}, receiver);
    quad(s, {-0.45f, 2, -0.45f}, {0.45f, 2, -0.45f}, {0.45f, 2, 0.45f}, {-0.45f, 2, 0.45f},
         area_light);
    quad(s, {-0.8f, 1, -0.8f}, {0.8f, 1, -0.8f}, {0.8f, 1, 0.8f}, {-0.8f, 1, 0.8f}, filter);
    quad(s, {-0.35f, 0.35f, -1.25f}, {0.35f, 0.35f, -1.25f}, {0.35f, 1.05f, -1.25f},
         {-0.35f, 1.05f, -1.25f}, card);
    quad(s, {-0.55f, 0.2f, 0.75f}, {0.55f, 0.2f, 0.75f}, {0.55f, 1.2f, 0.75f},
         {-0.55f, 1.2f, 0.75f}, clear);
    quad(s, {-0.55f, 0.2f, -0.2f}, {0.55f, 0.2f, -0.2f}, {0.55f, 1.2f, -0.2f},
         {-0.55f, 1.2f, -0.2f}, filter);
    camera(s, {0, 0.85f, 3.2f}, {0, 0.65f, -0.7f}, 38.0f);
}

// ---- asset scenes (scene/stanford_bunny.h, scene/stanford_dragon.h, scene/lux_cover.h;
// cameras app/render_runner.cpp:148-170).  Failures carry the reference's messages.

// load_obj_into_scene: the mesh and its placed instance; false when loading fails.
bool load_obj(SceneData& s, const std::filesystem::path& path, lux_obj_options o,
              std::string* error, const char* failure) {
    lux_obj_mesh* m = nullptr;
    if (lux_obj_load(path.string().c_str(), &o, &m) != LUX_OK) {
        std::fprintf(stderr, "OBJ error: %s\n", lux_last_error());
        *error = std::string(failure) + path.string();
        return false;
    }
    if (m) s.obj_meshes.push_back(m);
    return true;
}

// The loader's default material (Lambert 0.8) becomes thin Lambert, as the bunny and
// dragon scenes convert it.
bool grounded_asset(SceneData& s, const std::filesystem::path& path, lux_obj_options o,
                    std::string* error, const char* failure, const char* empty) {
    o.default_material = static_cast<int32_t>(s.materials.size());
    if (!load_obj(s, path, o, error, failure)) return false;
    if (s.obj_meshes.empty()) {
        *error = std::string(empty) + path.string();
        return false;
    }
    add_material(s, mat(kThinLambert, 0.8f, 0.8f, 0.8f));
    return true;
}

bool bunny(SceneData& s, const std::filesystem::path& root, std::string* error) {
    int floor = lambert(s, 0.5f, 0.5f, 0.5f);
    int light = emissive(s, 15.0f, 14.0f, 12.0f);
    quad(s, {-1, 0, 1}, {1, 0, 1}, {1, 0, -1}, {-1, 0, -1}, floor);
    quad(s, {-0.3f, 0.5f, -0.3f}, {0.3f, 0.5f, -0.3f}, {0.3f, 0.5f, 0.3f}, {-0.3f, 0.5f, 0.3f},
         light);
    lux_obj_options o{};
    o.ground_to_y = 1;
    if (!grounded_asset(s, root / "models" / "stanford-bunny.obj", o, error,
                        "Failed to load Stanford Bunny OBJ: ",
                        "Stanford Bunny OBJ loaded no triangles: "))
        return false;
    camera(s, {0.0f, 0.3f, 0.5f}, {-0.02f, 0.11f, 0.0f}, 40.0f);
    return true;
}

bool dragon(SceneData& s, const std::filesystem::path& root, std::string* error) {
    int floor = lambert(s, 0.5f, 0.5f, 0.5f);
    int light = emissive(s, 15.0f, 14.0f, 12.0f);
    quad(s, {-1, 0, 1}, {1, 0, 1}, {1, 0, -1}, {-1, 0, -1}, floor);
    quad(s, {-0.35f, 0.65f, -0.35f}, {0.35f, 0.65f, -0.35f}, {0.35f, 0.65f, 0.35f},
         {-0.35f, 0.65f, 0.35f}, light);
    lux_obj_options o{};
    o.scale_mode = LUX_OBJ_SCALE_MAX_EXTENT;
    o.target_extent = 0.5f;
    o.center_xz = 1;
    o.ground_to_y = 1;
    if (!grounded_asset(s, root / "models" / "dragon.obj", o, error,
                        "Failed to load dragon OBJ: ", "Dragon OBJ loaded no triangles: "))
        return false;
    camera(s, {0.0f, 0.35f, 0.8f}, {0.0f, 0.14f, 0.0f}, 42.0f);
    return true;
}

bool lux_cover(SceneData& s, const std::filesystem::path& root, std::string* error) {
    int floor = lambert(s, 0.42f, 0.43f, 0.42f);
    int key = emissive(s, 22.0f, 21.0f, 19.0f);
    s.materials[key].emission_two_sided = 1;
    int l = lambert(s, 0.78f, 0.76f, 0.70f);
    int u = add_material(s, mat(kDielectric, 0.90f, 0.97f, 1.00f, 0, 0, 0, 0.0f, 0.0f, 1.5f));
    int x = add_material(s, mat(kGgx, 0.82f, 0.78f, 0.68f, 0, 0, 0, 0.22f, 1.0f));
    quad(s, {-2.1f, 0, 0.18f}, {2.1f, 0, 0.18f}, {2.1f, 0, -2.2f}, {-2.1f, 0, -2.2f}, floor);
    quad(s, {-2.1f, 0, 0.18f}, {-2.1f, 1.8f, 0.18f}, {2.1f, 1.8f, 0.18f}, {2.1f, 0, 0.18f}, floor);
    quad(s, {-1.25f, 1.85f, -0.55f}, {1.25f, 1.85f, -0.55f}, {1.25f, 1.85f, 0.80f},
         {-1.25f, 1.85f, 0.80f}, key);
    const char* names[3] = {"L_lambert", "U_glass", "X_metal"};
    const int32_t ids[3] = {l, u, x};
    lux_obj_options o{};
    o.normal_mode = LUX_OBJ_NORMALS_SMOOTH;
    o.scale_mode = LUX_OBJ_SCALE_X_EXTENT;
    o.target_extent = 1.85f;
    o.center_xz = 1;
    o.ground_to_y = 1;
    o.binding_names = names;
    o.binding_ids = ids;
    o.binding_count = 3;
    o.default_material = -1;
    const std::filesystem::path path = root / "models" / "LUX.obj";
    if (!load_obj(s, path, o, error, "Failed to load LUX cover OBJ: ")) return false;
    if (s.obj_meshes.empty()) {
        *error = "LUX cover OBJ loaded no triangles: " + path.string();
        return false;
    }
    camera(s, {0.0f, 0.52f, -3.0f}, {0.0f, 0.36f, 0.0f}, 32.0f);
    return true;
}

// resolve_demo_asset_root (app/render_runner.cpp:37-79): assets/ next to the executable,
// else ./assets; the first candidate when neither exists.
std::filesystem::path asset_root(const char* argv0) {
    std::error_code ec;
    std::filesystem::path exe = std::filesystem::absolute(argv0, ec);
    if (ec) exe = argv0;
    std::filesystem::path dir = exe.parent_path();
    if (dir.empty()) dir = std::filesystem::current_path();
    std::filesystem::path candidates[2] = {dir / "assets", std::filesystem::current_path() / "assets"};
    for (const auto& c : candidates)
        if (std::filesystem::is_directory(c, ec) && !ec) return c;
    return candidates[0];
}

struct SceneEntry {
    const char* name;
    void (*make)(SceneData&);
    bool (*make_asset)(SceneData&, const std::filesystem::path&, std::string*);
};
constexpr SceneEntry kScenes[] = {
    {"cornell", cornell, nullptr},         {"direct-light", direct_light, nullptr},
    {"point-light", point_light, nullptr}, {"distant-light", distant_light, nullptr},
    {"uniform-env", uniform_env, nullptr}, {"transparent-filter", transparent_filter, nullptr},
    {"image-env", image_env, nullptr},     {"bunny", nullptr, bunny},
    {"dragon", nullptr, dragon},           {"lux-cover", nullptr, lux_cover},
};

double ms_since(Clock::time_point t) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
}

bool ends_with(const std::string& s, const char* suffix) {
    size_t n = std::strlen(suffix);
    return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

// resolve_output_paths / run_directory_output_path (app/render_runner.cpp:213-237).
std::string output_path(const Config& c) {
    if (c.output_mode == 1) return c.output;
    std::filesystem::path run(c.output_mode == 2 ? c.output : c.scene);
    std::string stem = run.filename().string();
    if (stem.empty()) stem = "render";
    return (std::filesystem::path("out") / run / (stem + ".ppm")).string();
}

int check(int status, const char* what) {
    if (status != LUX_OK) std::fprintf(stderr, "%s failed: %s\n", what, lux_last_error());
    return status;
}

}  // namespace

int main(int argc, char** argv) {
    auto total = Clock::now();
    Config c;
    if (!parse(argc, argv, c)) {
        usage(argv[0]);
        return 1;
    }
    if (c.help) {
        usage(argv[0]);
        return 0;
    }
    if (c.unsupported_option) {
        std::fprintf(stderr, "%s is not supported by this build\n", c.unsupported_name.c_str());
        return 1;
    }
    double t_setup = 0, t_gpu = 0, t_render = 0, t_write = 0;
    const SceneEntry* entry = nullptr;
    for (const SceneEntry& e : kScenes)
        if (c.scene == e.name) entry = &e;
    if (!entry) {
        std::string names;
        for (const SceneEntry& e : kScenes) names += (names.empty() ? "" : ", ") + std::string(e.name);
        std::fprintf(stderr, "Unknown scene '%s'. Available scenes: %s\n", c.scene.c_str(),
                     names.c_str());
        return 1;
    }
    if (!c.gpu) std::printf("Rendering on the GPU (the only path of this build)\n");
    auto t0 = Clock::now();
    SceneData data;
    if (entry->make) {
        entry->make(data);
    } else {
        std::string error;
        if (!entry->make_asset(data, asset_root(argv[0]), &error)) {
            std::fprintf(stderr, "Scene setup failed: %s\n", error.c_str());
            return 1;
        }
    }
    float aspect = static_cast<float>(c.width) / static_cast<float>(c.height);
    lux_scene_desc desc{};
    lux_mesh_desc mesh{};
    mesh.vertices = data.vertices.data();
    mesh.vertex_count = static_cast<int32_t>(data.vertices.size() / 3);
    mesh.indices = data.indices.data();
    mesh.material_ids = data.material_ids.data();
    mesh.triangle_count = static_cast<int32_t>(data.material_ids.size());
    lux_instance_desc inst{};
    inst.mesh = 0;
    inst.material_override = -1;
    const float identity[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    std::memcpy(inst.object_to_world, identity, sizeof(identity));
    // The default mesh and its instance first, then each loaded mesh with its placement
    // (scene-triangle order: instances in creation order).
    std::vector<lux_mesh_desc> meshes{mesh};
    std::vector<lux_instance_desc> instances{inst};
    for (lux_obj_mesh* m : data.obj_meshes) {
        lux_mesh_desc md{};
        md.vertices = m->vertices;
        md.normals = m->normals;
        md.uvs = m->uvs;
        md.vertex_count = m->vertex_count;
        md.indices = m->indices;
        md.material_ids = m->material_ids;
        md.triangle_count = m->triangle_count;
        lux_instance_desc id{};
        id.mesh = static_cast<int32_t>(meshes.size());
        id.material_override = -1;
        std::memcpy(id.object_to_world, m->object_to_world, sizeof(id.object_to_world));
        meshes.push_back(md);
        instances.push_back(id);
    }
    desc.materials = data.materials.data();
    desc.material_count = static_cast<int32_t>(data.materials.size());
    desc.meshes = meshes.data();
    desc.mesh_count = static_cast<int32_t>(meshes.size());
    desc.instances = instances.data();
    desc.instance_count = static_cast<int32_t>(instances.size());
    desc.lights = data.lights.empty() ? nullptr : data.lights.data();
    desc.light_count = static_cast<int32_t>(data.lights.size());
    for (size_t k = 0; k < data.images.size(); ++k) data.images[k].pixels = data.image_pixels[k].data();
    desc.images = data.images.empty() ? nullptr : data.images.data();
    desc.image_count = static_cast<int32_t>(data.images.size());
    if (check(lux_camera_perspective(data.cam_origin, data.cam_look_at, data.cam_vfov, aspect,
                                     0.0f, 1.0f, &desc.camera),
              "Scene setup"))
        return 1;
    t_setup = ms_since(t0);

    t0 = Clock::now();
    lux_ctx* ctx = nullptr;
    lux_scene* scene = nullptr;
    if (check(lux_ctx_create(&ctx, 0, nullptr), "GPU scene preparation")) return 1;
    if (check(lux_scene_create(ctx, &desc, &scene), "GPU scene preparation")) {
        lux_ctx_destroy(ctx);
        return 1;
    }
    t_gpu = ms_since(t0);
    std::printf("Built GPU TLAS/BLAS: %d TLAS nodes, %d instances, %d meshes\n",
                2 * desc.instance_count - 1, desc.instance_count, desc.mesh_count);

    lux_render_request req{};
    req.width = c.width;
    req.height = c.height;
    req.spp = c.spp;
    req.max_depth = c.max_depth;
    req.seed = 0;
    req.frame_index = 0;
    req.sample_offset = 0;
    req.light_sampler = c.light_sampler;
    std::vector<float> film(static_cast<size_t>(c.width) * c.height * 3);
    t0 = Clock::now();
    const bool aovs = (c.aov_mask & (kAovShadow | kAovNg | kAovNs)) != 0;
    std::vector<float> aov_shadow, aov_ng, aov_ns;
    for (auto [bit, image] : {std::pair{kAovShadow, &aov_shadow}, std::pair{kAovNg, &aov_ng},
                              std::pair{kAovNs, &aov_ns}})
        if (c.aov_mask & bit) image->assign(film.size(), 0.0f);
    auto ptr_of = [](std::vector<float>& v) { return v.empty() ? nullptr : v.data(); };
    int st = aovs ? lux_render_aovs(ctx, scene, &req, film.data(), ptr_of(aov_shadow), ptr_of(aov_ng),
                                    ptr_of(aov_ns))
                  : lux_render(ctx, scene, &req, film.data());
    t_render = ms_since(t0);
    if (check(st, "GPU render")) {
        lux_scene_destroy(scene);
        lux_ctx_destroy(ctx);
        return 1;
    }
    std::printf("GPU render-only time: %.3f ms\n", t_render);

    t0 = Clock::now();
    std::string path = output_path(c);
    std::filesystem::path parent = std::filesystem::path(path).parent_path();
    if (!parent.empty()) std::filesystem::create_directories(parent);
    bool pfm = ends_with(path, ".pfm");
    std::ofstream out(path, std::ios::binary);
    if (pfm) {
        std::vector<float> px(film.size());
        st = lux_film_encode(ctx, film.data(), c.width, c.height, c.spp, LUX_FILM_PFM, px.data());
        out << "PF\n" << c.width << " " << c.height << "\n-1.0\n";
        out.write(reinterpret_cast<const char*>(px.data()), px.size() * sizeof(float));
    } else {
        std::vector<unsigned char> px(film.size());
        st = lux_film_encode(ctx, film.data(), c.width, c.height, c.spp, LUX_FILM_PPM8, px.data());
        out << "P6\n" << c.width << " " << c.height << "\n255\n";
        out.write(reinterpret_cast<const char*>(px.data()), px.size());
    }
    out.close();
    if (!st && aovs) {
        std::printf("Wrote %s (%dx%d, %d spp, depth %d)\n", path.c_str(), c.width, c.height,
                    c.spp, c.max_depth);
        // write_debug_pixels (app/render_runner.cpp:250-256): PFM, else a linear PPM.
        const std::string prefix = c.debug_output.empty() ? path : c.debug_output;
        const struct {
            unsigned bit;
            const char* name;
            const char* label;
            std::vector<float>* image;
        } outs[] = {{kAovShadow, "shadow", "shadow classification", &aov_shadow},
                    {kAovNg, "ng", "geometric normal", &aov_ng},
                    {kAovNs, "ns", "shading normal", &aov_ns}};
        for (const auto& o : outs) {
            if (!(c.aov_mask & o.bit) || st) continue;
            const std::string apath = aov_path(prefix, o.name);
            std::filesystem::path aparent = std::filesystem::path(apath).parent_path();
            if (!aparent.empty()) std::filesystem::create_directories(aparent);
            std::ofstream f(apath, std::ios::binary);
            if (ends_with(apath, ".pfm")) {
                std::vector<float> px(film.size());
                st = lux_film_encode(ctx, o.image->data(), c.width, c.height, c.spp, LUX_FILM_PFM,
                                     px.data());
                f << "PF\n" << c.width << " " << c.height << "\n-1.0\n";
                f.write(reinterpret_cast<const char*>(px.data()), px.size() * sizeof(float));
            } else {
                std::vector<unsigned char> px(film.size());
                st = lux_film_encode(ctx, o.image->data(), c.width, c.height, c.spp,
                                     LUX_FILM_PPM8_LINEAR, px.data());
                f << "P6\n" << c.width << " " << c.height << "\n255\n";
                f.write(reinterpret_cast<const char*>(px.data()), px.size());
            }
            std::printf("Wrote %s (GPU %s AOV)\n", apath.c_str(), o.label);
        }
    }
    t_write = ms_since(t0);
    lux_scene_destroy(scene);
    lux_ctx_destroy(ctx);
    if (check(st, "Output write")) return 1;
    if (!aovs)
        std::printf("Wrote %s (%dx%d, %d spp, depth %d)\n", path.c_str(), c.width, c.height,
                    c.spp, c.max_depth);
    if (c.timing) {  // print_timing_breakdown (app/render_runner.cpp:270-285)
        std::printf("Timing breakdown:\n");
        std::printf("  scene setup: %.3f ms\n", t_setup);
        std::printf("  GPU scene preparation: %.3f ms\n", t_gpu);
        std::printf("  render: %.3f ms\n", t_render);
        std::printf("  output write: %.3f ms\n", t_write);
        std::printf("  total: %.3f ms\n", ms_since(total));
    }
    return 0;
}
