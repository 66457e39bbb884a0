/*
 * FP64 high-spp oracle of the path tracer (test infrastructure: only tests and the
 * bench's baseline legs load it; nothing in the product does).
 *
 * The estimator of the reference CPU tracer, trace_path
 * (integrator/cpu_path_tracer.cpp:403-498, with trace_shadow :27-73 and
 * estimate_direct_light :122-158), evaluated in double precision so that its
 * high-sample mean is the reference image up to Monte Carlo error only:
 *   - camera: pinhole rays through jittered pixel positions (generate_camera_ray,
 *     camera/camera.h:141-153; render_cpu_path_tracer :519-528);
 *   - emission on hits, single-sided unless two-sided, cos > 1e-7
 *     (material/material.h:125-134), MIS-weighted against light sampling after a
 *     non-delta bounce (path_transport.cuh:45-56, power heuristic,
 *     sampler/sample_record.h:50-57);
 *   - next-event estimation for Lambert, thin Lambert and GGX: one light picked with
 *     probability proportional to power, a uniform point on an area light
 *     (light/light_sampler.h:361-390), shadow rays through pass-through surfaces;
 *   - BSDFs of material/bsdf.h:93-529: Lambert, thin Lambert (50/50 reflect/transmit),
 *     GGX with VNDF sampling plus a diffuse lobe, dielectric (Fresnel, discrete),
 *     interface and transparent pass-through;
 *   - Russian roulette after depth 2 with p = min(0.95, max(T) * eta^2)
 *     (path_transport.cuh:58-84); ray offsets of 1e-5 (core/constants.h:11).
 * Only the expectation matters here, so the oracle draws its own random numbers
 * (SplitMix64, Steele, Lea and Flood 2014, keyed by seed, pixel and sample), selects
 * lights by its own power weights, and intersects through its own median-split BVH
 * in double.  Lights: area lights are the emissive triangles; point, distant and
 * uniform-infinite lights come from the light list.  Shading normals are the face
 * normals (the scenes it is used on carry none).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EPS 1e-5
#define EMIT_COS_EPS 1e-7
#define PI 3.14159265358979323846

typedef struct { double x, y, z; } d3;
static inline d3 v(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 vadd(d3 a, d3 b) { return v(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 vsub(d3 a, d3 b) { return v(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 vmul(d3 a, d3 b) { return v(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline d3 vs(d3 a, double s) { return v(a.x * s, a.y * s, a.z * s); }
static inline d3 vneg(d3 a) { return v(-a.x, -a.y, -a.z); }
static inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 cross(d3 a, d3 b) {
    return v(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline double len(d3 a) { return sqrt(dot(a, a)); }
static inline d3 norm(d3 a) { double l = len(a); return l > 0 ? vs(a, 1.0 / l) : a; }
static inline double maxc(d3 a) { return fmax(a.x, fmax(a.y, a.z)); }

/* ---------------------------------------------------------------- RNG */
typedef struct { uint64_t s; } Rng;
static inline uint64_t splitmix(uint64_t* s) {
    uint64_t z = (*s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static inline double rnd(Rng* r) { return (double)(splitmix(&r->s) >> 11) * (1.0 / 9007199254740992.0); }

/* ---------------------------------------------------------------- scene */
enum { LAMBERT = 0, THIN_LAMBERT = 1, GGX = 2, DIELECTRIC = 3, INTERFACE = 4, TRANSPARENT = 5 };
enum { M_NONE = 0, M_SOLID = 1, M_DISCRETE = 3 };
enum { F_DIFFUSE = 1, F_GLOSSY = 2, F_DREFL = 4, F_DTRANS = 8, F_TRANS = 16 };

typedef struct {
    int type, two_sided;
    d3 albedo, emission;
    double roughness, metallic, eta;
} Mat;

typedef struct { d3 v0, v1, v2, ng; double area; int mat; } Tri;

typedef struct {
    int kind;      /* 0 area, 1 point, 2 distant, 3 uniform infinite */
    int tri;
    d3 value, vec;
    double weight;
} Light;

typedef struct { double lo[3], hi[3]; int left, right, first, count; } Node;

typedef struct {
    Tri* tris;
    int ntri;
    int* order;
    Node* nodes;
    int nnodes;
    Mat* mats;
    int nmat;
    Light* lights;
    int nlights;
    double* cdf;
    double total;
    int* tri_light;
    d3 cam_o, cam_ll, cam_h, cam_v;
} Scene;

static double tri_axis(const Tri* t, int a) {
    const double* p0 = &t->v0.x; const double* p1 = &t->v1.x; const double* p2 = &t->v2.x;
    return (p0[a] + p1[a] + p2[a]) / 3.0;
}

static const Scene* g_sort_scene;
static int g_sort_axis;
static int cmp_centroid(const void* a, const void* b) {
    double ca = tri_axis(&g_sort_scene->tris[*(const int*)a], g_sort_axis);
    double cb = tri_axis(&g_sort_scene->tris[*(const int*)b], g_sort_axis);
    return ca < cb ? -1 : ca > cb ? 1 : 0;
}

static int build_node(Scene* s, int first, int count) {
    int id = s->nnodes++;
    Node* n = &s->nodes[id];
    for (int a = 0; a < 3; ++a) { n->lo[a] = INFINITY; n->hi[a] = -INFINITY; }
    double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = first; i < first + count; ++i) {
        const Tri* t = &s->tris[s->order[i]];
        const d3* vv[3] = {&t->v0, &t->v1, &t->v2};
        for (int k = 0; k < 3; ++k) {
            const double* p = &vv[k]->x;
            for (int a = 0; a < 3; ++a) { n->lo[a] = fmin(n->lo[a], p[a]); n->hi[a] = fmax(n->hi[a], p[a]); }
        }
        for (int a = 0; a < 3; ++a) {
            double c = tri_axis(t, a);
            clo[a] = fmin(clo[a], c); chi[a] = fmax(chi[a], c);
        }
    }
    if (count <= 4) {
        n->first = first; n->count = count; n->left = n->right = -1;
        return id;
    }
    int axis = 0;
    for (int a = 1; a < 3; ++a) if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
    g_sort_scene = s; g_sort_axis = axis;
    qsort(s->order + first, (size_t)count, sizeof(int), cmp_centroid);
    int half = count / 2;
    n->count = 0;
    int l = build_node(s, first, half);
    int r = build_node(s, first + half, count - half);
    s->nodes[id].left = l;
    s->nodes[id].right = r;
    return id;
}

static int box_hit(const Node* n, d3 o, d3 inv, const int par[3], double tmin, double tmax) {
    const double* oo = &o.x; const double* ii = &inv.x;
    for (int a = 0; a < 3; ++a) {
        if (par[a]) {
            if (oo[a] < n->lo[a] || oo[a] > n->hi[a]) return 0;
            continue;
        }
        double t0 = (n->lo[a] - oo[a]) * ii[a], t1 = (n->hi[a] - oo[a]) * ii[a];
        if (t0 > t1) { double t = t0; t0 = t1; t1 = t; }
        tmin = fmax(tmin, t0); tmax = fmin(tmax, t1);
        if (tmin > tmax) return 0;
    }
    return 1;
}

static int tri_hit(const Tri* t, d3 o, d3 d, double tmin, double tmax, double* tout) {
    d3 e1 = vsub(t->v1, t->v0), e2 = vsub(t->v2, t->v0);
    d3 p = cross(d, e2);
    double det = dot(e1, p);
    if (fabs(det) < 1e-300) return 0;
    double inv = 1.0 / det;
    d3 s = vsub(o, t->v0);
    double u = dot(s, p) * inv;
    if (u < 0 || u > 1) return 0;
    d3 q = cross(s, e1);
    double w = dot(d, q) * inv;
    if (w < 0 || u + w > 1) return 0;
    double tt = dot(e2, q) * inv;
    if (!(tt > tmin && tt < tmax)) return 0;
    *tout = tt;
    return 1;
}

/* Closest hit skipping triangle `skip`; returns the triangle or -1. */
static int intersect(const Scene* s, d3 o, d3 d, double tmin, double* tmax, int skip) {
    d3 inv; int par[3];
    const double* dd = &d.x; double* ii = &inv.x;
    for (int a = 0; a < 3; ++a) { par[a] = fabs(dd[a]) < 1e-300; ii[a] = par[a] ? 0 : 1.0 / dd[a]; }
    int stack[128], sp = 0, best = -1;
    if (s->nnodes == 0) return -1;
    stack[sp++] = 0;
    while (sp > 0) {
        const Node* n = &s->nodes[stack[--sp]];
        if (!box_hit(n, o, inv, par, tmin, *tmax)) continue;
        if (n->left < 0) {
            for (int i = n->first; i < n->first + n->count; ++i) {
                int k = s->order[i];
                double t;
                if (k != skip && tri_hit(&s->tris[k], o, d, tmin, *tmax, &t)) { *tmax = t; best = k; }
            }
        } else if (sp + 2 <= 128) {
            stack[sp++] = n->right;
            stack[sp++] = n->left;
        }
    }
    return best;
}

/* ---------------------------------------------------------------- BSDFs */
typedef struct { d3 wi, weight; double pdf, eta; int measure, flags; } Bs;
typedef struct { d3 p, ng, ns, wo; } It;

static d3 tangent(d3 n) { return fabs(n.x) > 0.9 ? norm(cross(v(0, 0, 1), n)) : norm(cross(v(1, 0, 0), n)); }
static d3 cos_hemi(d3 n, double ux, double uy) {
    double r = sqrt(ux), phi = 2 * PI * uy;
    double x = r * cos(phi), z = r * sin(phi), y = sqrt(fmax(0.0, 1 - ux));
    d3 t = tangent(n), b = cross(n, t);
    return norm(vadd(vadd(vs(t, x), vs(n, y)), vs(b, z)));
}
static int same_hemi(d3 n, d3 a, d3 b) { return dot(n, a) * dot(n, b) > 0; }
static d3 orient(d3 n, d3 ref) { return dot(n, ref) < 0 ? vneg(n) : n; }

static double clamp01(double x) { return fmax(0.0, fmin(1.0, x)); }
static d3 ggx_f0(const Mat* m) { double t = clamp01(m->metallic); return vadd(vs(v(0.04, 0.04, 0.04), 1 - t), vs(m->albedo, t)); }
static double ggx_dscale(const Mat* m) { return (1 - clamp01(m->metallic)) * fmax(0.0, 1 - maxc(ggx_f0(m))); }
static double ggx_alpha(const Mat* m) { double r = fmax(m->roughness, 0.02); return fmax(r * r, 1e-4); }
static double ggx_D(d3 h, d3 n, double a) {
    double c = dot(n, h); if (c <= 0) return 0;
    double a2 = a * a, den = c * c * (a2 - 1) + 1;
    return a2 / (PI * den * den);
}
static double ggx_G1(d3 w, d3 n, double a) {
    double c = dot(n, w); if (c <= 0) return 0;
    double t2 = (1 - c * c) / (c * c);
    return 2 / (1 + sqrt(1 + a * a * t2));
}
static double ggx_lambda(d3 w, d3 n, double a) {
    double c = dot(n, w); if (c <= 0) return 0;
    double t2 = fmax(0.0, 1 - c * c) / (c * c);
    return (sqrt(1 + a * a * t2) - 1) * 0.5;
}
static d3 schlick(d3 f0, double c) {
    double p = pow(1 - clamp01(c), 5);
    return vadd(f0, vs(vsub(v(1, 1, 1), f0), p));
}
static void ggx_lobes(const Mat* m, double* pd, double* ps) {
    int dv = maxc(m->albedo) > 0 && ggx_dscale(m) > 0, sv = maxc(ggx_f0(m)) > 0;
    if (sv && clamp01(m->metallic) >= 1 - 1e-4) { *pd = 0; *ps = 1; return; }
    if (dv && sv) { *pd = 0.5; *ps = 0.5; return; }
    if (dv) { *pd = 1; *ps = 0; return; }
    if (sv) { *pd = 0; *ps = 1; return; }
    *pd = *ps = 0;
}
static d3 ggx_spec_f(const Mat* m, const It* it, d3 wi) {
    d3 n = it->ns, wo = it->wo;
    if (dot(n, wo) <= 0 || dot(n, wi) <= 0) return v(0, 0, 0);
    d3 h = norm(vadd(wo, wi));
    double a = ggx_alpha(m);
    double D = ggx_D(h, n, a), G = 1 / (1 + ggx_lambda(wo, n, a) + ggx_lambda(wi, n, a));
    double den = 4 * dot(n, wo) * dot(n, wi);
    if (den <= 0) return v(0, 0, 0);
    return vs(schlick(ggx_f0(m), dot(wo, h)), D * G / den);
}
static double ggx_spec_pdf(const Mat* m, const It* it, d3 wi) {
    d3 n = it->ns, wo = it->wo;
    if (dot(n, wo) <= 0 || dot(n, wi) <= 0) return 0;
    d3 h = norm(vadd(wo, wi));
    double a = ggx_alpha(m), cwo = fabs(dot(n, wo)), woh = fabs(dot(wo, h));
    if (cwo <= 0 || woh <= 0) return 0;
    return ggx_D(h, n, a) * ggx_G1(wo, n, a) * woh / cwo / (4 * woh);
}
static d3 vndf(d3 wo, d3 n, double a, double ux, double uy) {
    d3 t = tangent(n), b = cross(n, t);
    d3 wl = v(dot(wo, t), dot(wo, b), dot(wo, n));
    d3 wh = norm(v(a * wl.x, a * wl.y, wl.z));
    if (wh.z < 0) wh = vneg(wh);
    d3 t1 = wh.z < 0.99999 ? norm(cross(v(0, 0, 1), wh)) : v(1, 0, 0);
    d3 t2 = cross(wh, t1);
    double r = sqrt(ux), phi = 2 * PI * uy;
    double px = r * cos(phi), py = r * sin(phi);
    double hh = sqrt(fmax(0.0, 1 - px * px)), blend = (1 + wh.z) * 0.5;
    py = (1 - blend) * hh + blend * py;
    double pz = sqrt(fmax(0.0, 1 - px * px - py * py));
    d3 nh = vadd(vadd(vs(t1, px), vs(t2, py)), vs(wh, pz));
    d3 ml = norm(v(a * nh.x, a * nh.y, fmax(1e-6, nh.z)));
    d3 wm = norm(vadd(vadd(vs(t, ml.x), vs(b, ml.y)), vs(n, ml.z)));
    return dot(wm, n) < 0 ? vneg(wm) : wm;
}

static d3 bsdf_f(const Mat* m, const It* it, d3 wi) {
    switch (m->type) {
        case LAMBERT: return same_hemi(it->ns, it->wo, wi) ? vs(m->albedo, 1 / PI) : v(0, 0, 0);
        case THIN_LAMBERT: return vs(m->albedo, 0.5 / PI);
        case GGX: {
            d3 diff = (dot(it->ns, it->wo) <= 0 || dot(it->ns, wi) <= 0) ? v(0, 0, 0)
                      : vs(m->albedo, ggx_dscale(m) / PI);
            return vadd(diff, ggx_spec_f(m, it, wi));
        }
        default: return v(0, 0, 0);
    }
}
static double bsdf_pdf(const Mat* m, const It* it, d3 wi) {
    double lam = same_hemi(it->ns, it->wo, wi) ? fabs(dot(it->ns, wi)) / PI : 0;
    switch (m->type) {
        case LAMBERT: return lam;
        case THIN_LAMBERT: return 0.5 * fabs(dot(it->ns, wi)) / PI;
        case GGX: { double pd, ps; ggx_lobes(m, &pd, &ps); return pd * lam + ps * ggx_spec_pdf(m, it, wi); }
        default: return 0;
    }
}
static void finish(Bs* s, const Mat* m, const It* it) {
    d3 f = bsdf_f(m, it, s->wi);
    s->pdf = bsdf_pdf(m, it, s->wi);
    s->measure = s->pdf > 0 ? M_SOLID : M_NONE;
    double c = fabs(dot(it->ns, s->wi));
    s->weight = (s->pdf > 0 && c > 0 && maxc(f) > 0) ? vs(f, c / s->pdf) : v(0, 0, 0);
}
static double fresnel(double ci, double ei, double et) {
    double si = sqrt(fmax(0.0, 1 - ci * ci)), st = ei / et * si;
    if (st >= 1) return 1;
    double ct = sqrt(fmax(0.0, 1 - st * st));
    double rpa = (et * ci - ei * ct) / (et * ci + ei * ct), rpe = (ei * ci - et * ct) / (ei * ci + et * ct);
    return (rpa * rpa + rpe * rpe) * 0.5;
}
static Bs sample_bsdf(const Mat* m, const It* it, double ux, double uy) {
    Bs s; memset(&s, 0, sizeof s); s.eta = 1;
    switch (m->type) {
        case LAMBERT:
            s.wi = cos_hemi(orient(it->ns, it->wo), ux, uy); s.flags = F_DIFFUSE; finish(&s, m, it); return s;
        case THIN_LAMBERT: {
            int refl = ux < 0.5;
            double rx = refl ? ux * 2 : (ux - 0.5) * 2;
            d3 side = orient(it->ns, it->wo);
            s.wi = cos_hemi(refl ? side : vneg(side), rx, uy);
            s.flags = refl ? F_DIFFUSE : (F_DIFFUSE | F_TRANS);
            finish(&s, m, it);
            return s;
        }
        case GGX: {
            if (dot(it->ns, it->wo) <= 0) return s;
            double pd, ps; ggx_lobes(m, &pd, &ps);
            if (pd <= 0 && ps <= 0) return s;
            if (pd > 0 && (ux < pd || ps <= 0)) {
                s.wi = cos_hemi(it->ns, ux / pd, uy); s.flags = F_DIFFUSE;
            } else {
                d3 h = vndf(it->wo, it->ns, ggx_alpha(m), (ux - pd) / ps, uy);
                s.wi = norm(vsub(vs(h, 2 * dot(it->wo, h)), it->wo));
                if (dot(it->ns, s.wi) <= 0 || ggx_spec_pdf(m, it, s.wi) <= 0) return s;
                s.flags = F_GLOSSY;
            }
            finish(&s, m, it);
            return s;
        }
        case DIELECTRIC: {
            double c = dot(it->wo, it->ns);
            int entering = c > 0;
            double ei = entering ? 1 : m->eta, et = entering ? m->eta : 1;
            d3 nn = entering ? it->ns : vneg(it->ns);
            c = fabs(c);
            double fr = fresnel(c, ei, et);
            s.measure = M_DISCRETE;
            double st = ei / et * sqrt(fmax(0.0, 1 - c * c));
            if (ux < fr || st >= 1) {
                s.wi = norm(vsub(vs(nn, 2 * c), it->wo));
                s.weight = m->albedo; s.pdf = ux < fr ? fr : 1; s.flags = F_DREFL;
                return s;
            }
            double ct = sqrt(fmax(0.0, 1 - st * st)), ratio = ei / et;
            s.wi = norm(vadd(vs(vneg(it->wo), ratio), vs(nn, ratio * c - ct)));
            double etap = et / ei;
            s.weight = vs(m->albedo, 1 / (etap * etap));
            s.pdf = 1 - fr; s.eta = etap; s.flags = F_DTRANS | F_TRANS;
            return s;
        }
        default:
            s.wi = norm(vneg(it->wo));
            s.weight = m->type == TRANSPARENT ? m->albedo : v(1, 1, 1);
            s.pdf = 1; s.measure = M_DISCRETE; s.flags = F_DTRANS | F_TRANS;
            return s;
    }
}

static int passthrough(const Mat* m) { return m->type == INTERFACE || m->type == TRANSPARENT; }
static int scattering(const Mat* m) {
    if (m->type == LAMBERT || m->type == THIN_LAMBERT) return maxc(m->albedo) > 0;
    return m->type == GGX || m->type == DIELECTRIC;
}
static int direct_lobe(const Mat* m) { return m->type == LAMBERT || m->type == THIN_LAMBERT || m->type == GGX; }
static double emit_cos(d3 ng, d3 wo, int two) {
    double c = dot(ng, wo);
    if (two) c = fabs(c);
    return c > EMIT_COS_EPS ? c : 0;
}
static double power_h(double a, double b) {
    if (a <= 0) return 0;
    double a2 = a * a, b2 = fmax(0.0, b); b2 *= b2;
    return a2 + b2 > 0 ? a2 / (a2 + b2) : 0;
}
static double pmf(const Scene* s, int i) { return s->total > 0 ? s->lights[i].weight / s->total : 0; }

static double area_pdf_sa(const Scene* s, int li, d3 pos, d3 ref) {
    const Light* L = &s->lights[li];
    const Tri* t = &s->tris[L->tri];
    d3 to = vsub(pos, ref);
    double d2 = dot(to, to);
    if (d2 <= EPS * EPS || t->area <= 0) return 0;
    d3 wi = vs(to, 1 / sqrt(d2));
    double c = emit_cos(t->ng, vneg(wi), s->mats[t->mat].two_sided);
    if (c <= 0) return 0;
    return pmf(s, li) * (d2 / t->area) / c;
}
static double inf_pdf(const Scene* s) {
    double p = 0;
    for (int i = 0; i < s->nlights; ++i) if (s->lights[i].kind == 3) p += pmf(s, i) / (4 * PI);
    return p;
}
static d3 inf_le(const Scene* s) {
    d3 le = v(0, 0, 0);
    for (int i = 0; i < s->nlights; ++i) if (s->lights[i].kind == 3) le = vadd(le, s->lights[i].value);
    return le;
}

/* Shadow transmittance from o along d over (EPS, tmax), through pass-through surfaces. */
static d3 shadow(const Scene* s, d3 o, d3 d, double tmax, int skip) {
    d3 tr = v(1, 1, 1);
    for (int seg = 0; seg < 1024; ++seg) {
        double t = tmax;
        int k = intersect(s, o, d, EPS, &t, skip);
        if (k < 0) return tr;
        const Mat* m = &s->mats[s->tris[k].mat];
        if (!passthrough(m)) return v(0, 0, 0);
        if (m->type == TRANSPARENT) tr = vmul(tr, m->albedo);
        if (maxc(tr) <= 0) return tr;
        double adv = t + EPS;
        if (adv >= tmax) return tr;
        o = vadd(o, vs(d, adv));
        tmax -= adv;
        skip = -1;
    }
    return v(0, 0, 0);
}

static d3 trace(const Scene* s, d3 o, d3 d, Rng* r, int max_depth) {
    d3 L = v(0, 0, 0), thr = v(1, 1, 1), prev_pos = v(0, 0, 0);
    double prev_pdf = 0, eta = 1;
    int prev_measure = M_NONE, prev_flags = 0, depth = 0;
    double tmin = EPS;
    for (int step = 0; step <= max_depth; ++step) {
        double t = INFINITY;
        int k = intersect(s, o, d, tmin, &t, -1);
        if (k < 0) {
            d3 le = inf_le(s);
            if (maxc(le) > 0) {
                if (depth == 0 || (prev_flags & (F_DREFL | F_DTRANS))) L = vadd(L, vmul(thr, le));
                else if (prev_measure == M_SOLID && prev_pdf > 0)
                    L = vadd(L, vs(vmul(thr, le), power_h(prev_pdf, inf_pdf(s))));
            }
            break;
        }
        const Tri* tri = &s->tris[k];
        const Mat* m = &s->mats[tri->mat];
        d3 pos = vadd(o, vs(d, t)), ng = tri->ng, wo = vneg(d);
        if (maxc(m->emission) > 0 && emit_cos(ng, wo, m->two_sided) > 0) {
            if (depth == 0 || (prev_flags & (F_DREFL | F_DTRANS))) L = vadd(L, vmul(thr, m->emission));
            else if (prev_measure == M_SOLID && prev_pdf > 0) {
                double lp = s->tri_light[k] >= 0 ? area_pdf_sa(s, s->tri_light[k], pos, prev_pos) : 0;
                L = vadd(L, vs(vmul(thr, m->emission), power_h(prev_pdf, lp)));
            }
        }
        if (passthrough(m)) {
            if (m->type == TRANSPARENT) thr = vmul(thr, m->albedo);
            if (maxc(thr) <= 0) break;
            o = vadd(pos, vs(d, EPS));
            tmin = EPS;
            continue;
        }
        if (!scattering(m) || step >= max_depth || depth >= max_depth) break;
        It it = {pos, ng, ng, wo};
        if (direct_lobe(m) && s->nlights > 0 && s->total > 0) {
            double su = rnd(r), ux = rnd(r), uy = rnd(r);
            int li = 0;
            double target = su * s->total;
            int lo = 0, hi = s->nlights - 1;
            while (lo < hi) { int mid = (lo + hi) / 2; if (s->cdf[mid] > target) hi = mid; else lo = mid + 1; }
            li = lo;
            const Light* Lt = &s->lights[li];
            double p = pmf(s, li);
            d3 wi = v(0, 0, 0), rad = v(0, 0, 0), lpos = v(0, 0, 0);
            double lpdf = 0, dist = INFINITY;
            int discrete = 0, ok = 0;
            if (Lt->kind == 0) {
                const Tri* lt = &s->tris[Lt->tri];
                double sq = sqrt(ux);
                lpos = vadd(vadd(vs(lt->v0, 1 - sq), vs(lt->v1, sq * (1 - uy))), vs(lt->v2, sq * uy));
                d3 to = vsub(lpos, pos);
                double d2 = dot(to, to);
                if (d2 > EPS * EPS) {
                    dist = sqrt(d2); wi = vs(to, 1 / dist);
                    double c = emit_cos(lt->ng, vneg(wi), s->mats[lt->mat].two_sided);
                    if (c > 0 && lt->area > 0) {
                        rad = s->mats[lt->mat].emission;
                        lpdf = p * (d2 / lt->area) / c;
                        ok = maxc(rad) > 0;
                    }
                }
            } else if (Lt->kind == 1) {
                d3 to = vsub(Lt->vec, pos);
                double d2 = dot(to, to);
                if (d2 > EPS * EPS) {
                    dist = sqrt(d2); wi = vs(to, 1 / dist); lpos = Lt->vec;
                    rad = vs(Lt->value, 1 / d2); lpdf = p; discrete = 1; ok = maxc(rad) > 0;
                }
            } else if (Lt->kind == 2) {
                wi = norm(Lt->vec); rad = Lt->value; lpdf = p; discrete = 1; ok = maxc(rad) > 0;
            } else {
                double z = 1 - 2 * ux, rr = sqrt(fmax(0.0, 1 - z * z)), phi = 2 * PI * uy;
                wi = v(rr * cos(phi), z, rr * sin(phi));
                rad = Lt->value; lpdf = p / (4 * PI); ok = maxc(rad) > 0;
            }
            if (ok && lpdf > 0) {
                d3 f = bsdf_f(m, &it, wi);
                double cs = fabs(dot(it.ns, wi));
                if (maxc(f) > 0 && cs > 0) {
                    d3 contrib = vs(vmul(f, rad), cs / lpdf);
                    double w = discrete ? 1 : power_h(lpdf, bsdf_pdf(m, &it, wi));
                    d3 so = vadd(pos, vs(dot(wi, ng) >= 0 ? ng : vneg(ng), EPS));
                    d3 sd = wi;
                    double smax = INFINITY;
                    int go = 1;
                    if (dist < INFINITY) {
                        d3 to = vsub(lpos, so);
                        double dd = len(to);
                        if (dd <= EPS) go = 0; else { sd = vs(to, 1 / dd); smax = dd - EPS; }
                    }
                    if (go) {
                        d3 tr = shadow(s, so, sd, smax, k);
                        if (maxc(tr) > 0) L = vadd(L, vmul(thr, vs(vmul(contrib, tr), w)));
                    }
                }
            }
        }
        Bs b = sample_bsdf(m, &it, rnd(r), rnd(r));
        if (b.pdf <= 0 || maxc(b.weight) <= 0) break;
        d3 nthr = vmul(thr, b.weight);
        double neta = eta * (((b.flags & (F_TRANS | F_DTRANS)) && b.eta > 0) ? b.eta * b.eta : 1);
        if (depth > 2) {
            double prob = fmin(0.95, maxc(nthr) * neta);
            if (!(rnd(r) <= prob) || prob <= 0) break;
            nthr = vs(nthr, 1 / prob);
        }
        thr = nthr; eta = neta;
        prev_pdf = b.pdf; prev_measure = b.measure; prev_flags = b.flags; prev_pos = pos;
        o = vadd(pos, vs(dot(b.wi, ng) >= 0 ? ng : vneg(ng), EPS));
        d = b.wi;
        tmin = EPS;
        ++depth;
    }
    return L;
}

/* ---------------------------------------------------------------- driver */
typedef struct {
    const Scene* s;
    int width, height, spp, depth, x0, y0, x1, y1;
    uint64_t seed;
    double *mean, *var;
    int next_row;
    pthread_mutex_t mu;
} Job;

static void* worker(void* arg) {
    Job* j = (Job*)arg;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        int y = j->next_row++;
        pthread_mutex_unlock(&j->mu);
        if (y >= j->y1) break;
        for (int x = j->x0; x < j->x1; ++x) {
            int pixel = y * j->width + x;
            double sum[3] = {0, 0, 0}, sq[3] = {0, 0, 0};
            for (int sidx = 0; sidx < j->spp; ++sidx) {
                Rng r;
                r.s = j->seed * 0x9e3779b97f4a7c15ULL ^ ((uint64_t)pixel << 24) ^ (uint64_t)sidx;
                (void)splitmix(&r.s);
                double u = (x + rnd(&r)) / j->width;
                double vv = (j->height - 1 - y + rnd(&r)) / j->height;
                d3 target = vadd(vadd(j->s->cam_ll, vs(j->s->cam_h, u)), vs(j->s->cam_v, vv));
                d3 dir = norm(vsub(target, j->s->cam_o));
                d3 c = trace(j->s, j->s->cam_o, dir, &r, j->depth);
                const double* cc = &c.x;
                for (int a = 0; a < 3; ++a) { sum[a] += cc[a]; sq[a] += cc[a] * cc[a]; }
            }
            int idx = (y - j->y0) * (j->x1 - j->x0) + (x - j->x0);
            for (int a = 0; a < 3; ++a) {
                double mu = sum[a] / j->spp;
                j->mean[3 * idx + a] = mu;
                j->var[3 * idx + a] = j->spp > 1 ? (sq[a] - j->spp * mu * mu) / (j->spp - 1) : 0;
            }
        }
    }
    return NULL;
}

/*
 * tris: n x 9 world-space floats; mids: n; mats: nmat x 11 (type, albedo3, emission3,
 * roughness, metallic, eta, two_sided); lights: nl x 7 (kind, vec3, value3);
 * cam: origin3, lower_left3, horizontal3, vertical3 (the pinhole camera's frame).
 * Writes the per-pixel mean radiance and its per-sample variance over the pixel
 * rectangle [x0, x1) x [y0, y1), row-major within the rectangle.
 */
int pt64_render(const float* tris, int ntri, const int* mids, const float* mats, int nmat,
                const float* lights, int nl, const float* cam, int width, int height, int spp,
                int max_depth, uint64_t seed, int x0, int y0, int x1, int y1, int threads,
                double* mean, double* var) {
    Scene s;
    memset(&s, 0, sizeof s);
    s.ntri = ntri;
    s.tris = (Tri*)calloc((size_t)(ntri > 0 ? ntri : 1), sizeof(Tri));
    s.order = (int*)calloc((size_t)(ntri > 0 ? ntri : 1), sizeof(int));
    s.nodes = (Node*)calloc((size_t)(2 * (ntri > 0 ? ntri : 1)), sizeof(Node));
    s.mats = (Mat*)calloc((size_t)(nmat > 0 ? nmat : 1), sizeof(Mat));
    s.tri_light = (int*)malloc(sizeof(int) * (size_t)(ntri > 0 ? ntri : 1));
    s.lights = (Light*)calloc((size_t)(ntri + nl + 1), sizeof(Light));
    s.cdf = (double*)calloc((size_t)(ntri + nl + 1), sizeof(double));
    s.nmat = nmat;
    for (int i = 0; i < nmat; ++i) {
        const float* f = mats + 11 * i;
        Mat* m = &s.mats[i];
        m->type = (int)f[0];
        m->albedo = v(f[1], f[2], f[3]);
        m->emission = v(f[4], f[5], f[6]);
        m->roughness = f[7]; m->metallic = f[8]; m->eta = f[9]; m->two_sided = f[10] != 0;
    }
    for (int i = 0; i < ntri; ++i) {
        const float* t = tris + 9 * i;
        Tri* tr = &s.tris[i];
        tr->v0 = v(t[0], t[1], t[2]); tr->v1 = v(t[3], t[4], t[5]); tr->v2 = v(t[6], t[7], t[8]);
        d3 c = cross(vsub(tr->v1, tr->v0), vsub(tr->v2, tr->v0));
        tr->ng = norm(c);
        tr->area = 0.5 * len(c);
        tr->mat = mids[i];
        s.order[i] = i;
        s.tri_light[i] = -1;
        const Mat* m = &s.mats[tr->mat];
        double lum = 0.2126 * m->emission.x + 0.7152 * m->emission.y + 0.0722 * m->emission.z;
        if (maxc(m->emission) > 0 && tr->area > 0) {
            Light* L = &s.lights[s.nlights];
            L->kind = 0; L->tri = i; L->weight = tr->area * fmax(1e-6, lum);
            s.tri_light[i] = s.nlights++;
        }
    }
    for (int i = 0; i < nl; ++i) {
        const float* f = lights + 7 * i;
        Light* L = &s.lights[s.nlights++];
        L->kind = (int)f[0];
        L->vec = v(f[1], f[2], f[3]);
        L->value = v(f[4], f[5], f[6]);
        L->weight = fmax(1e-6, 0.2126 * L->value.x + 0.7152 * L->value.y + 0.0722 * L->value.z);
    }
    for (int i = 0; i < s.nlights; ++i) { s.total += s.lights[i].weight; s.cdf[i] = s.total; }
    if (ntri > 0) build_node(&s, 0, ntri);
    s.cam_o = v(cam[0], cam[1], cam[2]);
    s.cam_ll = v(cam[3], cam[4], cam[5]);
    s.cam_h = v(cam[6], cam[7], cam[8]);
    s.cam_v = v(cam[9], cam[10], cam[11]);

    Job j;
    j.s = &s; j.width = width; j.height = height; j.spp = spp; j.depth = max_depth;
    j.x0 = x0; j.y0 = y0; j.x1 = x1; j.y1 = y1; j.seed = seed; j.mean = mean; j.var = var;
    j.next_row = y0;
    pthread_mutex_init(&j.mu, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    for (int i = 0; i < threads; ++i) pthread_create(&th[i], NULL, worker, &j);
    for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&j.mu);
    free(s.tris); free(s.order); free(s.nodes); free(s.mats); free(s.tri_light);
    free(s.lights); free(s.cdf);
    return 0;
}
