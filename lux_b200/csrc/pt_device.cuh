// Device functions of the wavefront path tracer: RNG, camera, BSDFs, light sampling,
// MIS / Russian roulette and the two-level scene traversal.
//
// Every function restates the reference's host/device code in the same arithmetic
// order (paths relative to the reference's src/); with contraction disabled
// (lux::mul/add/sub, and -fmad=false for the translation unit) a path computes the same
// values as the reference CPU tracer except where CUDA's sinf/cosf/powf round
// differently from the host libm (rare last-bit differences).
#pragma once

#include <cstdint>

#include "lux_bvh.cuh"
#include "lux_math.cuh"

namespace lux {
namespace pt {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 1.0f / kPi;
constexpr float kRayEpsilon = 1e-5f;          // core/constants.h:11
constexpr float kEmissionCosEpsilon = 1e-7f;  // material/material.h:27

// ------------------------------------------------------------------ vector helpers

LUX_HD f3 vdiv(f3 v, float s) {  // vec3::operator/ multiplies by 1/s (core/vec3.cuh:26)
    float inv = 1.0f / s;
    return f3{mul(v.x, inv), mul(v.y, inv), mul(v.z, inv)};
}
LUX_HD float length2(f3 v) { return dot(v, v); }
LUX_HD float length(f3 v) { return sqrtf(length2(v)); }
LUX_HD f3 normalize(f3 v) {  // core/vec3.cuh:62-66
    float len = length(v);
    return len > 0 ? vdiv(v, len) : v;
}
LUX_HD float max_component(f3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }
LUX_HD f3 splat(float s) { return f3{s, s, s}; }

// ------------------------------------------------------------------ RNG

// PCG-XSH-RR (core/pcg.cuh:11-41).
struct Pcg {
    uint64_t state;
    uint64_t inc;

    LUX_HD uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xorshifted = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = static_cast<uint32_t>(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
    }
    LUX_HD float next_float() {  // (next() >> 8) / 2^24
        return static_cast<float>(next() >> 8) / static_cast<float>(1 << 24);
    }
};

// make_render_sampler + make_sampler_state (integrator/render_context.h:37-54,
// sampler/sampler.h:165-176): seed' = seed ^ frame * golden; state seeded from
// (seed', pixel, sample), stream from (seed' >> 1) ^ (sample * 2891336453 + pixel).
LUX_HD Pcg make_sampler(uint64_t seed, int frame_index, int pixel, int sample) {
    uint64_t base = seed ^ (static_cast<uint64_t>(frame_index) * 0x9e3779b97f4a7c15ULL);
    uint64_t s = static_cast<uint64_t>(sample);
    uint64_t state = base + static_cast<uint64_t>(pixel) * 747796405ULL + s;
    uint64_t seq = (base >> 1) ^ (s * 2891336453ULL + static_cast<uint64_t>(pixel));
    Pcg p;
    p.state = 0;
    p.inc = (seq << 1u) | 1u;
    p.next();
    p.state += state;
    p.next();
    return p;
}

// ------------------------------------------------------------------ scene records

enum MaterialType : int {
    kLambert = 0,
    kThinLambert = 1,
    kGgx = 2,
    kDielectric = 3,
    kInterface = 4,
    kTransparent = 5,
};

struct Material {  // material/material.h:29-40
    int type;
    f3 albedo;
    f3 emission;
    int two_sided;
    float roughness;
    float metallic;
    float eta;
    int emission_image;   // image emission: scene image index; -1 constant emission
    f3 emission_scale;
};

LUX_HD bool is_scattering(const Material& m) {  // material/material.h:110-120
    switch (m.type) {
        case kLambert:
        case kThinLambert: return max_component(m.albedo) > 0;
        case kGgx:
        case kDielectric: return true;
        default: return false;
    }
}
LUX_HD bool is_passthrough(const Material& m) {
    return m.type == kInterface || m.type == kTransparent;
}
LUX_HD f3 passthrough_transmittance(const Material& m) {
    return m.type == kTransparent ? m.albedo : splat(1.0f);
}
LUX_HD bool has_direct_lighting_lobe(const Material& m) {
    return m.type == kLambert || m.type == kThinLambert || m.type == kGgx;
}

// emission_projected_cosine (material/material.h:125-134).
LUX_HD float emission_cosine(f3 ng, f3 wo, int two_sided) {
    float c = dot(ng, wo);
    if (!two_sided) return c > kEmissionCosEpsilon ? c : 0.0f;
    c = fabsf(c);
    return c > kEmissionCosEpsilon ? c : 0.0f;
}
LUX_HD f3 eval_emission(f3 emission, int two_sided, f3 ng, f3 wo) {
    if (max_component(emission) <= 0) return splat(0);
    if (emission_cosine(ng, wo, two_sided) <= 0) return splat(0);
    return emission;
}

// World-space triangle of one scene primitive (precomputed at upload with the same
// transform_point / transform_instance_normal arithmetic the reference applies per
// access, scene/gpu_scene_view.h:146-190).
struct alignas(16) SceneTri {
    float4 v0;  // xyz, material id (int bits)
    float4 v1;  // xyz, instance id (int bits)
    float4 v2;  // xyz, local triangle id (int bits)
};
struct alignas(16) SceneTriShading {
    float4 n0;  // xyz, u0
    float4 n1;  // xyz, v0
    float4 n2;  // xyz, u1
    float4 uv;  // v1, u2, v2, has_normals (1/0)
};

struct Instance {
    float m[12];     // object_to_world rows 0..2
    float inv[12];   // world_to_object rows 0..2
    int blas;        // mesh (BLAS) index
    int first_primitive;
};

struct Light {  // light/light.h:86-93 for the kinds this path supports
    int kind;              // 0 area, 1 point, 2 distant, 3 uniform infinite, 4 image infinite
    int primitive;         // area: scene triangle id; image infinite: index into env
    int two_sided;
    float area;
    f3 emission;           // area emission / point intensity / radiance / image scale
    f3 vec;                // point position / distant direction to light
    int image;             // area light with image emission: scene image index, else -1
    f3 image_scale;
};

// A scene image (SceneImageLightAsset pixels): RGB texels, row-major.
struct ImageView {
    const float* pixels;
    int width, height;
};

// Image infinite light (ImageInfiniteLight, light/light.h:79-87): latitude-longitude
// texels (RGB, unscaled) and the running sum of their sampling weights.
struct EnvLight {
    const float* pixels;   // width * height * 3
    const float* cdf;      // width * height
    int width, height;
    float total;
    f3 scale;
};

struct AliasEntry {  // light/light_distribution.h:22-26
    float probability;
    int alias;
    float pmf;
};

// LightBvhNode (light/light_distribution.h:33-40): a box around the lights below, their
// summed power, the children and parent (-1 none) and, in a leaf, the light's index.
struct LightNode {
    f3 lo;
    float power;
    f3 hi;
    int light;   // -1 in an internal node
    int left, right, parent, pad;
};

struct Camera {  // camera/camera.h:29-38 (perspective)
    f3 origin, lower_left, horizontal, vertical, lens_u, lens_v;
    float lens_radius;
};

struct SceneView {
    const Material* materials;
    int material_count;
    const SceneTri* tris;
    const SceneTriShading* shading;
    int primitive_count;
    const Instance* instances;
    int instance_count;
    BvhView tlas;
    const int* tlas_instance;  // TLAS sorted-input index -> instance id
    const BvhView* blas;       // one per mesh
    const Light* lights;
    int light_count;
    const EnvLight* env;             // image infinite lights, by Light::primitive
    const ImageView* images;         // scene images, for image emission
    float total_light_power;
    const AliasEntry* light_alias;   // power alias table, light_count entries
    int light_sampler;               // 0 uniform, 1 power
    // Light tree for the tree sampler (LightBvhTable, light/light_distribution.h:75-88):
    // area and point lights in the tree, the others (distant, infinite) in a power table
    // beside it.  light_tree is null when no light has bounds; the tree sampler then
    // picks by power.
    const LightNode* light_tree;
    int light_tree_count;
    int light_tree_root;
    const int* light_leaf;           // light index -> leaf node, -1 outside the tree
    const int* light_other_slot;     // light index -> slot of the other table, -1 none
    const int* other_lights;         // slot -> light index
    const AliasEntry* other_alias;   // alias table over the other lights' power
    int other_count;
    float other_power;
    const int* primitive_light;      // scene triangle -> light index (-1 none, -2 several)
    bool has_two_level;
    bool has_passthrough;            // some material is an interface or transparent filter
    Camera camera;
};

// ------------------------------------------------------------------ camera

// generate_camera_ray, perspective (camera/camera.h:141-153), pinhole or thin lens.
LUX_HD void camera_ray(const Camera& c, float u, float v, float lens_x, float lens_y, f3& o,
                       f3& d) {
    f3 target = (c.lower_left + c.horizontal * u) + c.vertical * v;
    o = c.origin;
    if (c.lens_radius > 0) {
        // concentric_sample_disk (camera/camera.h:60-75)
        float sx = sub(mul(2.0f, lens_x), 1.0f);
        float sy = sub(mul(2.0f, lens_y), 1.0f);
        float lx = 0, ly = 0;
        if (!(sx == 0 && sy == 0)) {
            float r, theta;
            if (fabsf(sx) > fabsf(sy)) {
                r = sx;
                theta = mul(kPi / 4.0f, sy / sx);
            } else {
                r = sy;
                theta = sub(kPi / 2.0f, mul(kPi / 4.0f, sx / sy));
            }
            lx = mul(r, cosf(theta));
            ly = mul(r, sinf(theta));
        }
        lx = mul(lx, c.lens_radius);
        ly = mul(ly, c.lens_radius);
        o = o + (c.lens_u * lx + c.lens_v * ly);
    }
    f3 dir = target - o;
    float len = length(dir);
    d = len > 0 ? vdiv(dir, len) : dir;
}

// ------------------------------------------------------------------ BSDFs (material/bsdf.h)

enum BsdfFlag : unsigned {
    kFlagDiffuse = 1u,
    kFlagGlossy = 2u,
    kFlagDeltaReflection = 4u,
    kFlagDeltaTransmission = 8u,
    kFlagTransmission = 16u,
};
LUX_HD bool is_delta(unsigned f) { return (f & (kFlagDeltaReflection | kFlagDeltaTransmission)) != 0; }
LUX_HD bool is_transmission(unsigned f) {
    return (f & (kFlagTransmission | kFlagDeltaTransmission)) != 0;
}

enum PdfMeasure : int { kMeasureNone = 0, kMeasureSolidAngle = 1, kMeasureArea = 2, kMeasureDiscrete = 3 };

struct BsdfSample {
    f3 wi = {0, 0, 0};
    f3 f = {0, 0, 0};
    f3 weight = {0, 0, 0};
    float pdf = 0;
    float eta = 1;
    int measure = kMeasureNone;
    unsigned flags = 0;
};

struct Interaction {
    f3 p, ng, ns, wo;
};

LUX_HD f3 make_tangent(f3 n) {  // bsdf.h:53-57
    return fabsf(n.x) > 0.9f ? normalize(cross(make_f3(0, 0, 1), n))
                             : normalize(cross(make_f3(1, 0, 0), n));
}

LUX_HD f3 cosine_sample_hemisphere(f3 n, float ux, float uy) {  // bsdf.h:59-69
    float radius = sqrtf(ux);
    float phi = mul(mul(2.0f, kPi), uy);
    float x = mul(radius, cosf(phi));
    float z = mul(radius, sinf(phi));
    float y = sqrtf(fmaxf(0.0f, sub(1.0f, ux)));
    f3 t = make_tangent(n);
    f3 b = cross(n, t);
    return normalize((t * x + n * y) + b * z);
}

LUX_HD bool same_hemisphere(f3 n, f3 a, f3 b) { return mul(dot(n, a), dot(n, b)) > 0; }
LUX_HD float abs_cosine(f3 n, f3 d) { return fabsf(dot(n, d)); }
LUX_HD f3 orient(f3 n, f3 ref) { return dot(n, ref) < 0 ? -n : n; }

LUX_HD void finalize_smooth(BsdfSample& s, const Interaction& it) {  // bsdf.h:79-89
    if (s.pdf > 0) s.measure = kMeasureSolidAngle;
    float c = abs_cosine(it.ns, s.wi);
    if (s.pdf > 0 && c > 0 && max_component(s.f) > 0) s.weight = s.f * (c / s.pdf);
}

LUX_HD f3 eval_lambert(const Material& m, const Interaction& it, f3 wi) {
    if (!same_hemisphere(it.ns, it.wo, wi)) return splat(0);
    return m.albedo * kInvPi;
}
LUX_HD float pdf_lambert(const Interaction& it, f3 wi) {
    if (!same_hemisphere(it.ns, it.wo, wi)) return 0;
    return mul(abs_cosine(it.ns, wi), kInvPi);
}
LUX_HD f3 eval_thin_lambert(const Material& m) { return m.albedo * mul(0.5f, kInvPi); }
LUX_HD float pdf_thin_lambert(const Interaction& it, f3 wi) {
    return mul(mul(0.5f, abs_cosine(it.ns, wi)), kInvPi);
}

LUX_HD BsdfSample sample_lambert(const Material& m, const Interaction& it, float ux, float uy) {
    BsdfSample s;  // bsdf.h:125-136
    f3 n = orient(it.ns, it.wo);
    s.wi = cosine_sample_hemisphere(n, ux, uy);
    s.f = eval_lambert(m, it, s.wi);
    s.pdf = pdf_lambert(it, s.wi);
    s.flags = kFlagDiffuse;
    finalize_smooth(s, it);
    return s;
}

LUX_HD BsdfSample sample_thin_lambert(const Material& m, const Interaction& it, float ux,
                                      float uy) {
    BsdfSample s;  // bsdf.h:138-152
    bool refl = ux < 0.5f;
    float rx = refl ? mul(ux, 2.0f) : mul(sub(ux, 0.5f), 2.0f);
    f3 wo_side = orient(it.ns, it.wo);
    f3 n = refl ? wo_side : -wo_side;
    s.wi = cosine_sample_hemisphere(n, rx, uy);
    s.f = eval_thin_lambert(m);
    s.pdf = pdf_thin_lambert(it, s.wi);
    s.flags = refl ? kFlagDiffuse : (kFlagDiffuse | kFlagTransmission);
    finalize_smooth(s, it);
    return s;
}

// GGX (bsdf.h:158-396).
LUX_HD float clamp01(float v) { return fmaxf(0.0f, fminf(1.0f, v)); }
LUX_HD float ggx_metallic(const Material& m) { return clamp01(m.metallic); }
LUX_HD f3 ggx_f0(const Material& m) {  // mix(0.04, albedo, metallic)
    float t = ggx_metallic(m);
    return splat(0.04f) * sub(1.0f, t) + m.albedo * t;
}
LUX_HD float ggx_diffuse_scale(const Material& m) {
    f3 f0 = ggx_f0(m);
    return mul(sub(1.0f, ggx_metallic(m)), fmaxf(0.0f, sub(1.0f, max_component(f0))));
}
LUX_HD float ggx_alpha(const Material& m) {
    float r = fmaxf(m.roughness, 0.02f);
    return fmaxf(mul(r, r), 1e-4f);
}
LUX_HD float ggx_d(f3 h, f3 n, float alpha) {
    float c = dot(n, h);
    if (c <= 0) return 0;
    float a2 = mul(alpha, alpha);
    float denom = add(mul(mul(c, c), sub(a2, 1.0f)), 1.0f);
    return a2 / mul(mul(kPi, denom), denom);
}
LUX_HD float ggx_g1(f3 v, f3 n, float alpha) {
    float c = dot(n, v);
    if (c <= 0) return 0;
    float a2 = mul(alpha, alpha);
    float tan2 = sub(1.0f, mul(c, c)) / mul(c, c);
    return 2.0f / add(1.0f, sqrtf(add(1.0f, mul(a2, tan2))));
}
LUX_HD float ggx_lambda(f3 v, f3 n, float alpha) {
    float c = dot(n, v);
    if (c <= 0) return 0;
    float c2 = mul(c, c);
    float tan2 = fmaxf(0.0f, sub(1.0f, c2)) / c2;
    return mul(sub(sqrtf(add(1.0f, mul(mul(alpha, alpha), tan2))), 1.0f), 0.5f);
}
LUX_HD float ggx_g(f3 wo, f3 wi, f3 n, float alpha) {
    return 1.0f / add(add(1.0f, ggx_lambda(wo, n, alpha)), ggx_lambda(wi, n, alpha));
}
LUX_HD f3 fresnel_schlick(f3 f0, float c) {
    c = clamp01(c);
    float p5 = powf(sub(1.0f, c), 5.0f);
    return f0 + (splat(1.0f) - f0) * p5;
}
LUX_HD f3 eval_ggx_diffuse(const Material& m, const Interaction& it, f3 wi) {
    if (dot(it.ns, it.wo) <= 0 || dot(it.ns, wi) <= 0) return splat(0);
    return m.albedo * mul(ggx_diffuse_scale(m), kInvPi);
}
LUX_HD f3 eval_ggx_specular(const Material& m, const Interaction& it, f3 wi) {
    f3 wo = it.wo, n = it.ns;
    if (dot(n, wo) <= 0 || dot(n, wi) <= 0) return splat(0);
    f3 h = normalize(wo + wi);
    float alpha = ggx_alpha(m);
    float d = ggx_d(h, n, alpha);
    float g = ggx_g(wo, wi, n, alpha);
    f3 fr = fresnel_schlick(ggx_f0(m), dot(wo, h));
    float denom = mul(mul(4.0f, dot(n, wo)), dot(n, wi));
    if (denom <= 0) return splat(0);
    return vdiv(fr * mul(d, g), denom);  // (D * G * F) / denom
}
LUX_HD float pdf_ggx_specular(const Material& m, const Interaction& it, f3 wi) {
    f3 wo = it.wo, n = it.ns;
    if (dot(n, wo) <= 0 || dot(n, wi) <= 0) return 0;
    f3 h = normalize(wo + wi);
    float alpha = ggx_alpha(m);
    float d = ggx_d(h, n, alpha);
    float cwo = fabsf(dot(n, wo));
    float woh = fabsf(dot(wo, h));
    if (cwo <= 0 || woh <= 0) return 0;
    float pdf_wm = mul(mul(d, ggx_g1(wo, n, alpha)), woh) / cwo;
    return pdf_wm / mul(4.0f, woh);
}
LUX_HD f3 sample_visible_normal(f3 wo, f3 n, float alpha, float ux, float uy) {
    f3 t = make_tangent(n);
    f3 b = cross(n, t);
    f3 wl = make_f3(dot(wo, t), dot(wo, b), dot(wo, n));
    f3 wh = normalize(make_f3(mul(alpha, wl.x), mul(alpha, wl.y), wl.z));
    if (wh.z < 0) wh = -wh;
    f3 t1 = wh.z < 0.99999f ? normalize(cross(make_f3(0, 0, 1), wh)) : make_f3(1, 0, 0);
    f3 t2 = cross(wh, t1);
    float r = sqrtf(ux);
    float phi = mul(2.0f * kPi, uy);
    float px = mul(r, cosf(phi));
    float py = mul(r, sinf(phi));
    float hh = sqrtf(fmaxf(0.0f, sub(1.0f, mul(px, px))));
    float blend = mul(add(1.0f, wh.z), 0.5f);
    py = add(mul(sub(1.0f, blend), hh), mul(blend, py));
    float pz = sqrtf(fmaxf(0.0f, sub(sub(1.0f, mul(px, px)), mul(py, py))));
    f3 nh = (t1 * px + t2 * py) + wh * pz;
    f3 ml = normalize(make_f3(mul(alpha, nh.x), mul(alpha, nh.y), fmaxf(1e-6f, nh.z)));
    f3 wm = normalize((t * ml.x + b * ml.y) + n * ml.z);
    return dot(wm, n) < 0 ? -wm : wm;
}
LUX_HD BsdfSample sample_ggx_specular(const Material& m, const Interaction& it, float ux,
                                      float uy) {
    BsdfSample s;
    f3 wo = it.wo, n = it.ns;
    if (dot(n, wo) <= 0) return s;
    float alpha = ggx_alpha(m);
    f3 h = sample_visible_normal(wo, n, alpha, ux, uy);
    s.wi = normalize(h * mul(2.0f, dot(wo, h)) - wo);
    if (dot(n, s.wi) <= 0) return s;
    s.f = eval_ggx_specular(m, it, s.wi);
    s.pdf = pdf_ggx_specular(m, it, s.wi);
    s.flags = kFlagGlossy;
    finalize_smooth(s, it);
    return s;
}
LUX_HD void ggx_lobes(const Material& m, float& pd, float& ps) {  // bsdf.h:340-354
    bool diffuse_valid = max_component(m.albedo) > 0 && ggx_diffuse_scale(m) > 0;
    bool specular_valid = max_component(ggx_f0(m)) > 0;
    if (specular_valid && ggx_metallic(m) >= sub(1.0f, 1e-4f)) { pd = 0; ps = 1; return; }
    if (diffuse_valid && specular_valid) { pd = 0.5f; ps = 0.5f; return; }
    if (diffuse_valid) { pd = 1; ps = 0; return; }
    if (specular_valid) { pd = 0; ps = 1; return; }
    pd = 0;
    ps = 0;
}
LUX_HD f3 eval_ggx(const Material& m, const Interaction& it, f3 wi) {
    return eval_ggx_diffuse(m, it, wi) + eval_ggx_specular(m, it, wi);
}
LUX_HD float pdf_ggx(const Material& m, const Interaction& it, f3 wi) {
    float pd, ps;
    ggx_lobes(m, pd, ps);
    return add(mul(pd, pdf_lambert(it, wi)), mul(ps, pdf_ggx_specular(m, it, wi)));
}
LUX_HD BsdfSample sample_ggx(const Material& m, const Interaction& it, float ux, float uy) {
    BsdfSample s;  // bsdf.h:371-396
    f3 n = it.ns;
    if (dot(n, it.wo) <= 0) return s;
    float pd, ps;
    ggx_lobes(m, pd, ps);
    if (pd <= 0 && ps <= 0) return s;
    if (pd > 0 && (ux < pd || ps <= 0)) {
        s.wi = cosine_sample_hemisphere(n, ux / pd, uy);
        s.flags = kFlagDiffuse;
    } else {
        BsdfSample spec = sample_ggx_specular(m, it, sub(ux, pd) / ps, uy);
        if (spec.pdf <= 0) return s;
        s.wi = spec.wi;
        s.flags = kFlagGlossy;
    }
    s.f = eval_ggx(m, it, s.wi);
    s.pdf = pdf_ggx(m, it, s.wi);
    finalize_smooth(s, it);
    return s;
}

// Dielectric (bsdf.h:402-474).
LUX_HD float fresnel_dielectric(float ci, float ei, float et) {
    float si = sqrtf(fmaxf(0.0f, sub(1.0f, mul(ci, ci))));
    float st = mul(ei / et, si);
    if (st >= 1.0f) return 1.0f;
    float ct = sqrtf(fmaxf(0.0f, sub(1.0f, mul(st, st))));
    float r_parl = sub(mul(et, ci), mul(ei, ct)) / add(mul(et, ci), mul(ei, ct));
    float r_perp = sub(mul(ei, ci), mul(et, ct)) / add(mul(ei, ci), mul(et, ct));
    return mul(add(mul(r_parl, r_parl), mul(r_perp, r_perp)), 0.5f);
}
LUX_HD BsdfSample sample_dielectric(const Material& m, const Interaction& it, float ux) {
    BsdfSample s;
    f3 wo = it.wo, n = it.ns;
    float c = dot(wo, n);
    bool entering = c > 0;
    float ei = entering ? 1.0f : m.eta;
    float et = entering ? m.eta : 1.0f;
    f3 nn = entering ? n : -n;
    c = fabsf(c);
    float fr = fresnel_dielectric(c, ei, et);
    if (ux < fr) {
        s.wi = normalize(nn * mul(2.0f, c) - wo);
        s.weight = m.albedo;
        s.pdf = fr;
        s.eta = 1.0f;
        s.measure = kMeasureDiscrete;
        s.flags = kFlagDeltaReflection;
        return s;
    }
    float st = mul(ei / et, sqrtf(fmaxf(0.0f, sub(1.0f, mul(c, c)))));
    if (st >= 1.0f) {
        s.wi = normalize(nn * mul(2.0f, c) - wo);
        s.weight = m.albedo;
        s.pdf = 1.0f;
        s.eta = 1.0f;
        s.measure = kMeasureDiscrete;
        s.flags = kFlagDeltaReflection;
        return s;
    }
    float ct = sqrtf(fmaxf(0.0f, sub(1.0f, mul(st, st))));
    float ratio = ei / et;
    s.wi = normalize((-wo) * ratio + nn * sub(mul(ratio, c), ct));
    float etap = et / ei;
    s.weight = vdiv(m.albedo, mul(etap, etap));
    s.pdf = sub(1.0f, fr);
    s.eta = etap;
    s.measure = kMeasureDiscrete;
    s.flags = kFlagDeltaTransmission | kFlagTransmission;
    return s;
}

LUX_HD f3 eval_bsdf(const Material& m, const Interaction& it, f3 wi) {
    switch (m.type) {
        case kLambert: return eval_lambert(m, it, wi);
        case kThinLambert: return eval_thin_lambert(m);
        case kGgx: return eval_ggx(m, it, wi);
        default: return splat(0);
    }
}
LUX_HD float pdf_bsdf(const Material& m, const Interaction& it, f3 wi) {
    switch (m.type) {
        case kLambert: return pdf_lambert(it, wi);
        case kThinLambert: return pdf_thin_lambert(it, wi);
        case kGgx: return pdf_ggx(m, it, wi);
        default: return 0;
    }
}
LUX_HD BsdfSample sample_bsdf(const Material& m, const Interaction& it, float ux, float uy) {
    switch (m.type) {
        case kLambert: return sample_lambert(m, it, ux, uy);
        case kThinLambert: return sample_thin_lambert(m, it, ux, uy);
        case kGgx: return sample_ggx(m, it, ux, uy);
        case kDielectric: return sample_dielectric(m, it, ux);
        default: {
            BsdfSample s;  // interface / transparent (bsdf.h:494-529)
            s.wi = normalize(-it.wo);
            s.weight = m.type == kTransparent ? m.albedo : splat(1.0f);
            s.pdf = 1.0f;
            s.measure = kMeasureDiscrete;
            s.flags = kFlagDeltaTransmission | kFlagTransmission;
            return s;
        }
    }
}

// ------------------------------------------------------------------ MIS / RR (path_transport.cuh)

LUX_HD float power_heuristic(float a_pdf, float b_pdf) {  // sampler/sample_record.h:50-57
    if (a_pdf <= 0) return 0;
    float a = mul(a_pdf, a_pdf);
    float b = fmaxf(0.0f, b_pdf);
    b = mul(b, b);
    float den = add(a, b);
    return den > 0 ? a / den : 0;
}

// ------------------------------------------------------------------ triangle helpers

LUX_HD f3 tri_v(const float4& p) { return make_f3(p.x, p.y, p.z); }

LUX_HD f3 triangle_normal(f3 v0, f3 v1, f3 v2) { return normalize(cross(v1 - v0, v2 - v0)); }
LUX_HD float triangle_area(f3 v0, f3 v1, f3 v2) {
    return mul(0.5f, length(cross(v1 - v0, v2 - v0)));
}

// interpolate_triangle_normal (scene/gpu_scene_view.h:209-217).
LUX_HD f3 shading_normal(const SceneTriShading& s, f3 face, float u, float v) {
    if (s.uv.w == 0.0f) return face;
    float w = sub(sub(1.0f, u), v);
    f3 n = (tri_v(s.n0) * w + tri_v(s.n1) * u) + tri_v(s.n2) * v;
    if (length2(n) == 0) return face;
    return normalize(n);
}

}  // namespace pt
}  // namespace lux
