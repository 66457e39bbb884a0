// Device code shared by the single-request wavefront renderer (wavefront.cu) and the
// multi-request server (server.cu): the SoA path pool, two-level traversal, light
// sampling, and the per-path stages (camera, extend, shade, shadow).
//
// Every stage restates the reference's per-path arithmetic (paths relative to src/):
// camera integrator/wavefront_kernels.cu:234-270 with the draw order of
// cpu_path_tracer.cpp:532-542; extend wavefront_kernels.cu:272-354; shade
// cpu_path_tracer.cpp:403-498 (emission + MIS, pass-through, NEE, BSDF sample, RR);
// shadow cpu_path_tracer.cpp:27-73.  A path's step count (extends so far) is its scatter
// depth plus its pass-through depth, so paths of different depths can share one queue.
#pragma once

#include <cuda_runtime.h>

#include "../../include/lux_gpu.h"
#include "lux_wide.cuh"
#include "pt_device.cuh"

namespace lux {
namespace pt {

constexpr int kThreads = 256;
constexpr int kStack = 72;
constexpr int kClasses = 5;       // Lambert, thin Lambert, GGX, dielectric, pass-through
constexpr int kShadowSegments = 1024;

// SoA path state and queues (capacity paths, 16-byte records).
struct PathPool {
    int capacity = 0;
    float4* thr_eta = nullptr;      // throughput.rgb, eta scale
    float4* rad = nullptr;          // radiance.rgb
    float4* prev = nullptr;         // previous sample reference position, pdf
    int4* meta = nullptr;           // pixel, sample, depth | passthrough << 16, measure | flags << 8
    uint4* rng = nullptr;           // PCG state lo/hi, inc lo/hi
    float4* ray_o = nullptr;        // origin, t_min
    float4* ray_d = nullptr;        // direction, t_max
    float4* hit = nullptr;          // t, u, v, primitive (int bits)
    float4* sh_o = nullptr;         // origin, t_max
    float4* sh_d = nullptr;         // direction, ignored primitive (int bits)
    float4* sh_c = nullptr;         // contribution.rgb, mis weight
    float4* sh_t = nullptr;         // throughput.rgb at the vertex
    int* qray[2] = {nullptr, nullptr};
    int* qmat = nullptr;            // kClasses * capacity
    int* qshadow = nullptr;
};

// Device buffers of a pool (wavefront.cu).
int path_pool_alloc(PathPool& pool, int capacity);
void path_pool_free(PathPool& pool);

namespace {

LUX_D unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Warp-aggregated append: lanes with the same queue share one atomic.
LUX_D int append(int* counter_base, int queue, bool active) {
    unsigned mask = __ballot_sync(0xffffffffu, active);
    if (!active) return -1;
    unsigned peers = __match_any_sync(mask, queue);
    int leader = __ffs(peers) - 1;
    int base = 0;
    if (static_cast<int>(threadIdx.x & 31) == leader) base = atomicAdd(counter_base + queue, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + __popc(peers & lanemask_lt());
}

LUX_D f3 xyz(const float4& v) { return make_f3(v.x, v.y, v.z); }

// ------------------------------------------------------------------ traversal

struct SceneHit {
    int prim = -1;
    float t = 0, u = 0, v = 0;
};

// transform_point / transform_vector with the implicit row (0 0 0 1)
// (core/mat4.cuh:173-199).
LUX_D f3 xform_point(const float* m, f3 p) {
    float x = add(add(add(mul(m[0], p.x), mul(m[1], p.y)), mul(m[2], p.z)), m[3]);
    float y = add(add(add(mul(m[4], p.x), mul(m[5], p.y)), mul(m[6], p.z)), m[7]);
    float z = add(add(add(mul(m[8], p.x), mul(m[9], p.y)), mul(m[10], p.z)), m[11]);
    float w = add(add(add(mul(0.0f, p.x), mul(0.0f, p.y)), mul(0.0f, p.z)), 1.0f);
    return w == 1.0f ? make_f3(x, y, z) : make_f3(x / w, y / w, z / w);
}
LUX_D f3 xform_vector(const float* m, f3 v) {
    return make_f3(add(add(mul(m[0], v.x), mul(m[1], v.y)), mul(m[2], v.z)),
                   add(add(mul(m[4], v.x), mul(m[5], v.y)), mul(m[6], v.z)),
                   add(add(mul(m[8], v.x), mul(m[9], v.y)), mul(m[10], v.z)));
}

// Node visits and triangle tests of a walk in the reference's visit order: each box the
// reference's stackless walk tests (the root's, and both children's of every node it
// enters: bvh/bvh_device.cuh:43-90) and each triangle it tests; instances: TLAS leaves
// whose BLAS was searched.  Filled only by the kCount variants below.
struct WalkCounts {
    unsigned long long boxes = 0, tris = 0, instances = 0;
};

// Closest hit inside one BLAS in object space, reference order (bvh/bvh_device.cuh:92-134
// with GpuMeshPrimitiveIntersector, scene/gpu_scene_bvh.cuh:15-42).  best_t enters as the
// current bound; returns the local triangle id or -1.  kCount adds to *wc.
template <bool kCount = false>
LUX_D int blas_closest(const BvhView& b, f3 o, f3 d, float tmin, float& best_t, float& bu,
                       float& bv, int ignored_local, int* error, WalkCounts* wc = nullptr) {
    if (b.n <= 0) return -1;
    ray3 r{o, tmin, d, best_t};
    slab_ray sr = make_slab_ray(r);
    float tn;
    if (kCount) wc->boxes += 1;
    if (!slab_hit(sr, load_root(b.root), best_t, tn)) return -1;
    int2 stack[kStack];  // (node ref, entry t bits): one 8-byte access per entry
    int sp = 0;
    int cur = b.n == 1 ? ~0 : 0;
    int best = -1;
    const long long bound = 2ll * b.n + 64;
    for (long long step = 0;; ++step) {
        if (step > bound || cur >= b.n - 1 || ~cur >= b.n) {
            atomicOr(error, kErrLoopBound);
            return -1;
        }
        bool pop = true;
        if (cur >= 0) {
            BvhNode nd = load_node(b.nodes, cur);
            float tl, tr;
            if (kCount) wc->boxes += 2;
            bool hl = slab_hit(sr, node_left_box(nd), best_t, tl);
            bool hr = slab_hit(sr, node_right_box(nd), best_t, tr);
            if (hl) {
                if (hr) {
                    if (sp >= kStack) {
                        atomicOr(error, kErrStackOverflow);
                        return -1;
                    }
                    stack[sp] = make_int2(nd.ch.y, __float_as_int(tr));
                    ++sp;
                }
                cur = nd.ch.x;
                pop = false;
            } else if (hr) {
                cur = nd.ch.y;
                pop = false;
            }
        } else {
            const float4* tp = reinterpret_cast<const float4*>(b.tris + ~cur);
            float4 p0 = __ldg(tp);
            int local = __float_as_int(p0.w);
            if (local != ignored_local) {
                if (kCount) wc->tris += 1;
                float4 p1 = __ldg(tp + 1);
                float4 p2 = __ldg(tp + 2);
                float t, u, v;
                if (moller_trumbore(o, d, xyz(p0), xyz(p1), xyz(p2), t, u, v) && t > tmin
                    && t < best_t) {
                    best = local;
                    best_t = t;
                    bu = u;
                    bv = v;
                }
            }
        }
        if (pop) {
            bool resumed = false;
            while (sp > 0) {
                --sp;
                const int2 e = stack[sp];
                if (!(__int_as_float(e.y) > best_t)) {
                    cur = e.x;
                    resumed = true;
                    break;
                }
            }
            if (!resumed) break;
        }
    }
    return best;
}

// Two-level closest hit (intersect_scene_bvh_device, scene/gpu_scene_bvh.cuh:44-135):
// TLAS over instance boxes in reference order; at each instance leaf the ray is taken
// to object space and its BLAS searched with t_max = the current best.  ignored: scene
// triangle id skipped (shadow rays leaving a surface), -1 none.  kCount adds the
// walk's node visits and triangle tests (both levels) to *wc.
template <bool kCount = false>
LUX_D SceneHit scene_closest(const SceneView& sc, f3 o, f3 d, float tmin, float tmax,
                             int ignored, int* error, WalkCounts* wc = nullptr) {
    SceneHit h;
    h.t = tmax;
    if (!sc.has_two_level) return h;
    const BvhView& tl = sc.tlas;
    ray3 r{o, tmin, d, tmax};
    slab_ray sr = make_slab_ray(r);
    float tn;
    if (kCount) wc->boxes += 1;
    if (!slab_hit(sr, load_root(tl.root), h.t, tn)) return h;
    int ign_instance = -1, ign_local = -1;
    if (ignored >= 0) {
        float4 v1 = __ldg(&sc.tris[ignored].v1);
        float4 v2 = __ldg(&sc.tris[ignored].v2);
        ign_instance = __float_as_int(v1.w);
        ign_local = __float_as_int(v2.w);
    }
    int2 stack[kStack];  // (node ref, entry t bits): one 8-byte access per entry
    int sp = 0;
    int cur = tl.n == 1 ? ~0 : 0;
    const long long bound = 2ll * tl.n + 64;
    for (long long step = 0;; ++step) {
        if (step > bound || cur >= tl.n - 1 || ~cur >= tl.n) {
            atomicOr(error, kErrLoopBound);
            return SceneHit{-1, tmax, 0, 0};
        }
        bool pop = true;
        if (cur >= 0) {
            BvhNode nd = load_node(tl.nodes, cur);
            float a, b;
            if (kCount) wc->boxes += 2;
            bool hl = slab_hit(sr, node_left_box(nd), h.t, a);
            bool hr = slab_hit(sr, node_right_box(nd), h.t, b);
            if (hl) {
                if (hr) {
                    if (sp >= kStack) {
                        atomicOr(error, kErrStackOverflow);
                        return SceneHit{-1, tmax, 0, 0};
                    }
                    stack[sp] = make_int2(nd.ch.y, __float_as_int(b));
                    ++sp;
                }
                cur = nd.ch.x;
                pop = false;
            } else if (hr) {
                cur = nd.ch.y;
                pop = false;
            }
        } else {
            int inst_id = sc.tlas_instance[tl.sorted_ids[~cur]];
            const Instance& inst = sc.instances[inst_id];
            f3 lo = xform_point(inst.inv, o);
            f3 ld = xform_vector(inst.inv, d);
            float best = h.t;
            float u = 0, v = 0;
            if (kCount) wc->instances += 1;
            int local = blas_closest<kCount>(sc.blas[inst.blas], lo, ld, tmin, best, u, v,
                                             inst_id == ign_instance ? ign_local : -1, error,
                                             wc);
            if (local >= 0 && best < h.t) {
                h.prim = inst.first_primitive + local;
                h.t = best;
                h.u = u;
                h.v = v;
            }
        }
        if (pop) {
            bool resumed = false;
            while (sp > 0) {
                --sp;
                const int2 e = stack[sp];
                if (!(__int_as_float(e.y) > h.t)) {
                    cur = e.x;
                    resumed = true;
                    break;
                }
            }
            if (!resumed) break;
        }
    }
    return h;
}

// scene_closest as a resumable walk: step() advances by one node visit or one triangle
// (or instance) test, followed by the pops it enables, so a kernel can interleave many
// walks per warp and refill lanes as walks finish.  The TLAS is walked over its binary
// nodes (a TLAS of at most kFlatTlas instances is entered leaf by leaf: init() tests every
// leaf box and defers the passing ones in leaf order), each BLAS over its quantised 4-wide
// nodes (lux_wide.cuh: every leaf the binary
// walk reaches is reached in the same left-first order and accepted by the exact test of
// its own box, the triangle's box formed from its record), so the leaves tested and the
// best hit after each are those of scene_closest / blas_closest above and the result is
// the same.  The stacks live apart from the scalar state, which then stays in registers.
constexpr int kWideBlasStack = 96;   // three deferred children per 4-wide level
constexpr int kFlatTlas = 4;          // TLAS leaves tested together when a walk starts

struct WalkStacks {  // deferred (node ref, entry t bits), TLAS and BLAS
    int2 t[kStack];
    int2 b[kWideBlasStack];
};

struct TwoLevelWalk {
    f3 o, d;
    float tmin;
    slab_ray sr;
    SceneHit hit;                 // best so far (hit.t is the current bound)
    int ign_instance, ign_local;
    int t_cur, t_sp;
    unsigned t_steps;             // steps of the walk (bounded by 2n + 64 per level)
    bool in_blas;
    const WideNode* b_wide;
    const TriRecord* b_tris;
    int b_n, b_cur, b_sp, b_ignored, b_first;
    unsigned b_steps;
    f3 lo, ld;
    slab_ray lsr;
    unsigned lneg;                // octant of the object-space ray (octant_ray::neg)
    bool done;
    bool any_hit;                 // end at the first accepted triangle (occlusion only)

    LUX_D void init(const SceneView& sc, WalkStacks& k, f3 ro, f3 rd, float rtmin, float rtmax,
                    int ignored, bool first_hit = false) {
        any_hit = first_hit;
        o = ro;
        d = rd;
        tmin = rtmin;
        hit = SceneHit{};
        hit.t = rtmax;
        in_blas = false;
        t_sp = 0;
        t_steps = 0;
        done = true;
        if (!sc.has_two_level) return;
        ign_instance = -1;
        ign_local = -1;
        if (ignored >= 0) {
            float4 v1 = __ldg(&sc.tris[ignored].v1);
            float4 v2 = __ldg(&sc.tris[ignored].v2);
            ign_instance = __float_as_int(v1.w);
            ign_local = __float_as_int(v2.w);
        }
        sr = make_slab_ray(ray3{o, tmin, d, rtmax});
        float tn;
        if (!slab_hit(sr, load_root(sc.tlas.root), hit.t, tn)) return;
        t_cur = sc.tlas.n == 1 ? ~0 : 0;
        done = false;
        const BvhView& tl = sc.tlas;
        if (tl.n >= 2 && tl.n <= kFlatTlas) {
            // A TLAS of a few instances: every leaf box is tested here, in leaf order (the
            // binary walk's left-first order), and the passing leaves after the first are
            // deferred with their entry t as the walk defers children, so the walk enters
            // the same instances under the same bounds without stepping through the
            // TLAS's internal nodes (a leaf box passes under a bound exactly when every
            // box above it does).
            int first = -1;
            float first_t = 0.0f;
            for (int j = tl.n - 1; j >= 0; --j) {
                float te;
                if (slab_hit(sr, leaf_box(tl, j), hit.t, te)) {
                    if (first >= 0) k.t[t_sp++] = make_int2(~first, __float_as_int(first_t));
                    first = j;
                    first_t = te;
                }
            }
            if (first < 0) {
                done = true;
                return;
            }
            t_cur = ~first;
        }
    }

    LUX_D void fail(int* error, int bit, float rtmax) {
        atomicOr(error, bit);
        hit = SceneHit{};
        hit.t = rtmax;
        done = true;
    }

    // Resumes the deepest deferred TLAS child that still passes; false when none is left.
    LUX_D bool pop_tlas(const WalkStacks& k) {
        while (t_sp > 0) {
            --t_sp;
            const int2 e = k.t[t_sp];
            if (!(__int_as_float(e.y) > hit.t)) {
                t_cur = e.x;
                return true;
            }
        }
        return false;
    }
    LUX_D bool pop_blas(const WalkStacks& k) {
        while (b_sp > 0) {
            --b_sp;
            const int2 e = k.b[b_sp];
            if (!(__int_as_float(e.y) > hit.t)) {
                b_cur = e.x;
                return true;
            }
        }
        return false;
    }

    // One step; returns true when the walk is complete (hit holds the result).
    LUX_D bool step(const SceneView& sc, WalkStacks& k, int* error) {
        if (done) return true;
        const BvhView& tl = sc.tlas;
        if (in_blas) {
            if (++b_steps > 2u * static_cast<unsigned>(b_n) + 64u || b_cur >= b_n - 1 ||
                ~b_cur >= b_n) {
                fail(error, kErrLoopBound, INFINITY);
                return true;
            }
            const octant_ray lorr{lsr.o, lsr.inv, lsr.tmin, lneg};
            bool pop = true;
            if (b_cur >= 0) {
                const WideNode w = load_wide(b_wide, b_cur);
                float tt[4];
                const unsigned m = wide_test(w, lsr, lorr, hit.t, tt);
                if (m) {
                    const int f = __ffs(m) - 1;
                    if (b_sp + __popc(m) - 1 > kWideBlasStack) {
                        fail(error, kErrStackOverflow, INFINITY);
                        return true;
                    }
#pragma unroll
                    for (int c = 3; c >= 1; --c) {
                        if (c > f && ((m >> c) & 1u)) {
                            k.b[b_sp] = make_int2(wide_ref(w, c), __float_as_int(tt[c]));
                            ++b_sp;
                        }
                    }
                    b_cur = wide_ref(w, f);
                    pop = false;
                }
            } else {
                const float4* tp = reinterpret_cast<const float4*>(b_tris + ~b_cur);
                const float4 p0 = __ldg(tp);
                const int local = __float_as_int(p0.w);
                if (local != b_ignored) {
                    const float4 p1 = __ldg(tp + 1);
                    const float4 p2 = __ldg(tp + 2);
                    float tn, t, u, v;
                    // The leaf's exact box (the triangle's box) under the current best t,
                    // then the triangle.
                    if (child_hit(triangle_box(xyz(p0), xyz(p1), xyz(p2)), lsr, lorr, hit.t, tn)
                        && moller_trumbore(lo, ld, xyz(p0), xyz(p1), xyz(p2), t, u, v)
                        && t > tmin && t < hit.t) {
                        hit.prim = b_first + local;
                        hit.t = t;
                        hit.u = u;
                        hit.v = v;
                        if (any_hit) {
                            done = true;
                            return true;
                        }
                    }
                }
            }
            if (pop && !pop_blas(k)) {
                in_blas = false;
                if (!pop_tlas(k)) done = true;
            }
            return done;
        }
        if (++t_steps > 2u * static_cast<unsigned>(tl.n) + 64u || t_cur >= tl.n - 1 ||
            ~t_cur >= tl.n) {
            fail(error, kErrLoopBound, INFINITY);
            return true;
        }
        bool pop = true;
        if (t_cur >= 0) {
            BvhNode nd = load_node(tl.nodes, t_cur);
            float a, b;
            bool hl = slab_hit(sr, node_left_box(nd), hit.t, a);
            bool hr = slab_hit(sr, node_right_box(nd), hit.t, b);
            if (hl) {
                if (hr) {
                    if (t_sp >= kStack) {
                        fail(error, kErrStackOverflow, INFINITY);
                        return true;
                    }
                    k.t[t_sp] = make_int2(nd.ch.y, __float_as_int(b));
                    ++t_sp;
                }
                t_cur = nd.ch.x;
                pop = false;
            } else if (hr) {
                t_cur = nd.ch.y;
                pop = false;
            }
        } else if (enter(sc)) {
            return false;
        }
        if (pop && !pop_tlas(k)) done = true;
        return done;
    }

    // Enters the instance of TLAS leaf ~t_cur: the ray in its object space and the BLAS
    // root's test; true when the walk goes on in the BLAS.
    LUX_D bool enter(const SceneView& sc) {
        const int inst_id = sc.tlas_instance[sc.tlas.sorted_ids[~t_cur]];
        const Instance& inst = sc.instances[inst_id];
        const BvhView& b = sc.blas[inst.blas];
        if (b.n <= 0) return false;
        lo = xform_point(inst.inv, o);
        ld = xform_vector(inst.inv, d);
        lsr = make_slab_ray(ray3{lo, tmin, ld, hit.t});
        float tn;
        if (!slab_hit(lsr, load_root(b.root), hit.t, tn)) return false;
        in_blas = true;
        lneg = make_octant_ray(lsr).neg;
        b_wide = b.wide;
        b_tris = b.tris;
        b_n = b.n;
        b_cur = b.n == 1 ? ~0 : 0;
        b_sp = 0;
        b_steps = 0;
        b_ignored = inst_id == ign_instance ? ign_local : -1;
        b_first = inst.first_primitive;
        return true;
    }
};

// ------------------------------------------------------------------ lights

// sample_alias_table_index (light/light_sampler.h:71-82).
LUX_D int sample_alias(const AliasEntry* table, int count, float u) {
    float scaled = mul(fminf(u, 0.99999994f), static_cast<float>(count));
    int column = static_cast<int>(scaled);
    if (column >= count) column = count - 1;
    float threshold = sub(scaled, static_cast<float>(column));
    const AliasEntry& e = table[column];
    int index = threshold < e.probability ? column : e.alias;
    return index >= 0 && index < count ? index : -1;
}

// ---- light tree (light/light_sampler.h:90-348).  Every walk is bounded by the node
// count, as the reference's.

// light_bvh_node_importance with squared_distance_to_bounds: power over the squared
// distance from p to the node's box, the distance kept at least kRayEpsilon.
LUX_D float light_node_importance(const SceneView& sc, int i, f3 p) {
    if (i < 0 || i >= sc.light_tree_count) return 0;
    const LightNode& n = sc.light_tree[i];
    if (n.power <= 0 || n.lo.x > n.hi.x || n.lo.y > n.hi.y || n.lo.z > n.hi.z) return 0;
    const float pa[3] = {p.x, p.y, p.z};
    const float lo[3] = {n.lo.x, n.lo.y, n.lo.z};
    const float hi[3] = {n.hi.x, n.hi.y, n.hi.z};
    float d2 = 0;
    for (int a = 0; a < 3; ++a) {
        float delta = 0;
        if (pa[a] < lo[a]) delta = sub(lo[a], pa[a]);
        else if (pa[a] > hi[a]) delta = sub(pa[a], hi[a]);
        d2 = add(d2, mul(delta, delta));
    }
    d2 = fmaxf(d2, mul(kRayEpsilon, kRayEpsilon));
    return n.power / d2;
}

// light_bvh_child_probability: the child's share of its parent's two importances.
LUX_D float light_child_probability(const SceneView& sc, int parent, int child, f3 p) {
    const int count = sc.light_tree_count;
    if (parent < 0 || parent >= count || child < 0 || child >= count) return 0;
    const LightNode& n = sc.light_tree[parent];
    if (child != n.left && child != n.right) return 0;
    const float l = light_node_importance(sc, n.left, p);
    const float r = light_node_importance(sc, n.right, p);
    const float total = add(l, r);
    if (total <= 0) return 0;
    const float lp = l / total;
    return child == n.left ? lp : sub(1.0f, lp);
}

// sample_light_bvh: root to leaf, the draw rescaled at each step.
LUX_D int sample_light_tree(const SceneView& sc, f3 p, float select_u, float& pmf) {
    pmf = 0;
    const int count = sc.light_tree_count;
    int node = sc.light_tree_root;
    if (!sc.light_tree || node < 0 || node >= count) return -1;
    float u = fminf(select_u, 0.99999994f);
    pmf = 1;
    for (int depth = 0; depth < count; ++depth) {
        const LightNode& n = sc.light_tree[node];
        if (n.light >= 0) return n.light;
        const float lp = light_child_probability(sc, node, n.left, p);
        if (lp <= 0) {
            node = n.right;
        } else if (lp >= 1) {
            node = n.left;
        } else if (u < lp) {
            pmf = mul(pmf, lp);
            u = u / lp;
            node = n.left;
        } else {
            const float rp = sub(1.0f, lp);
            pmf = mul(pmf, rp);
            u = sub(u, lp) / rp;
            node = n.right;
        }
        if (node < 0 || node >= count) {
            pmf = 0;
            return -1;
        }
    }
    pmf = 0;
    return -1;
}

// light_bvh_pmf: the product of child probabilities from the light's leaf to the root.
LUX_D float light_tree_pmf(const SceneView& sc, f3 p, int light) {
    const int count = sc.light_tree_count;
    if (!sc.light_tree || !sc.light_leaf || light < 0 || light >= sc.light_count) return 0;
    int node = sc.light_leaf[light];
    if (node < 0 || node >= count) return 0;
    float pmf = 1;
    for (int depth = 0; depth < count; ++depth) {
        const int parent = sc.light_tree[node].parent;
        if (parent < 0) return pmf;
        const float pr = light_child_probability(sc, parent, node, p);
        if (pr <= 0) return 0;
        pmf = mul(pmf, pr);
        node = parent;
        if (node >= count) return 0;
    }
    return 0;
}

// The tree's share of the total power and the other table's power
// (sample_light_bvh_mixture / light_bvh_mixture_pmf, light/light_sampler.h:265-359).
LUX_D bool light_tree_split(const SceneView& sc, float& tree_p, float& other) {
    const float tree_power = sc.light_tree[sc.light_tree_root].power;
    if (tree_power <= 0) return false;
    other = sc.other_count > 0 ? fmaxf(0.0f, sc.other_power) : 0.0f;
    const float total = add(tree_power, other);
    if (total <= 0) return false;
    tree_p = tree_power / total;
    return true;
}

// sample_indexed_discrete_light over the other table's alias entries.
LUX_D int sample_other_light(const SceneView& sc, float u, float& pmf) {
    pmf = 0;
    if (!sc.other_lights || !sc.other_alias || sc.other_count <= 0 || sc.other_power <= 0)
        return -1;
    const int slot = sample_alias(sc.other_alias, sc.other_count, u);
    if (slot < 0) return -1;
    pmf = sc.other_alias[slot].pmf;
    return pmf > 0 ? sc.other_lights[slot] : -1;
}

LUX_D int sample_light_mixture(const SceneView& sc, f3 p, float select_u, float& pmf) {
    pmf = 0;
    float tree_p, other;
    if (!light_tree_split(sc, tree_p, other)) return -1;
    if (other <= 0 || tree_p >= 1) return sample_light_tree(sc, p, select_u, pmf);
    if (tree_p <= 0) return sample_other_light(sc, select_u, pmf);
    const float u = fminf(select_u, 0.99999994f);
    float part = 0;
    int index;
    if (u < tree_p) {
        index = sample_light_tree(sc, p, u / tree_p, part);
        pmf = mul(tree_p, part);
    } else {
        const float other_p = sub(1.0f, tree_p);
        index = sample_other_light(sc, sub(u, tree_p) / other_p, part);
        pmf = mul(other_p, part);
    }
    return pmf > 0 ? index : -1;
}

LUX_D float light_mixture_pmf(const SceneView& sc, f3 p, int light) {
    float tree_p, other;
    if (light < 0 || !light_tree_split(sc, tree_p, other)) return 0;
    if (light < sc.light_count && sc.light_leaf[light] >= 0)
        return mul(tree_p, light_tree_pmf(sc, p, light));
    const int slot = light < sc.light_count && sc.light_other_slot ? sc.light_other_slot[light] : -1;
    if (slot < 0 || other <= 0 || !sc.other_alias) return 0;
    return mul(sub(1.0f, tree_p), sc.other_alias[slot].pmf);
}

LUX_D bool use_light_tree(const SceneView& sc, int sampler) {
    return sampler == 2 && sc.light_tree && sc.light_leaf && sc.light_tree_count > 0 &&
           sc.light_tree_root >= 0 && sc.light_tree_root < sc.light_tree_count;
}

// light_pmf (gpu_scene_light_sampler.cuh:9-45): the selection probability of a light at
// shading position p; p matters to the tree sampler only.
LUX_D float light_pmf(const SceneView& sc, int sampler, f3 p, int index) {
    if (index < 0 || index >= sc.light_count || sc.total_light_power <= 0) return 0;
    if (sampler == 0) return 1.0f / static_cast<float>(sc.light_count);
    if (use_light_tree(sc, sampler)) return light_mixture_pmf(sc, p, index);
    return sc.light_alias ? sc.light_alias[index].pmf : 0.0f;
}

// sample_scene_light (gpu_scene_light_sampler.cuh:47-96): the light picked by select_u
// at shading position p and its pmf (the tree walk's own, else light_pmf); -1 when none.
LUX_D int select_light(const SceneView& sc, int sampler, f3 p, float select_u, float& pmf) {
    pmf = 0;
    if (sc.light_count <= 0 || sc.total_light_power <= 0) return -1;
    int index;
    float selected = 0;
    if (sampler == 0) {
        index = static_cast<int>(mul(fminf(select_u, 0.99999994f), static_cast<float>(sc.light_count)));
        if (index >= sc.light_count) index = sc.light_count - 1;
    } else if (use_light_tree(sc, sampler)) {
        index = sample_light_mixture(sc, p, select_u, selected);
    } else {
        if (!sc.light_alias) return -1;
        index = sample_alias(sc.light_alias, sc.light_count, select_u);
    }
    if (index < 0) return -1;
    pmf = selected > 0 ? selected : light_pmf(sc, sampler, p, index);
    return index;
}

struct LightLi {
    f3 wi, position, radiance;
    float distance = INFINITY;
    float pdf = 0;
    int measure = kMeasureSolidAngle;
    bool valid = false;
};

LUX_D f3 sample_triangle_area(f3 v0, f3 v1, f3 v2, float ux, float uy) {  // light_sampler.h:361-367
    float s = sqrtf(ux);
    float b0 = sub(1.0f, s);
    float b1 = mul(s, sub(1.0f, uy));
    float b2 = mul(s, uy);
    return (v0 * b0 + v1 * b1) + v2 * b2;
}

LUX_D float solid_angle_pdf(f3 lpos, f3 lnormal, int two_sided, float pdf_area, f3 ref) {
    f3 to = lpos - ref;  // pdf_solid_angle (light/light_sampler.h:380-390)
    float d2 = length2(to);
    if (d2 <= mul(kRayEpsilon, kRayEpsilon) || pdf_area <= 0) return 0;
    f3 wi = vdiv(to, sqrtf(d2));
    float c = emission_cosine(lnormal, -wi, two_sided);
    if (c <= 0) return 0;
    return mul(pdf_area, d2) / c;
}

// ------------------------------------------------------------------ image infinite lights
// direction_to_latlong_uv / latlong_uv_to_direction / image_env_lookup /
// image_infinite_pdf_for_texel / sample_image_infinite_light / image_infinite_pdf
// (light/light.h:144-269).

LUX_D float2 env_uv(f3 wi) {
    f3 w = normalize(wi);
    float phi = atan2f(w.z, w.x);
    if (phi < 0) phi = add(phi, 2.0f * kPi);
    float theta = acosf(fmaxf(-1.0f, fminf(1.0f, w.y)));
    return make_float2(mul(phi, 0.5f * kInvPi), mul(theta, kInvPi));
}

LUX_D int env_texel(const EnvLight& e, float2 uv) {
    int x = static_cast<int>(fminf(static_cast<float>(e.width - 1), floorf(mul(uv.x, static_cast<float>(e.width)))));
    int y = static_cast<int>(fminf(static_cast<float>(e.height - 1), floorf(mul(uv.y, static_cast<float>(e.height)))));
    return y * e.width + x;
}

LUX_D f3 env_lookup(const EnvLight& e, f3 wi) {
    if (!e.pixels || e.width <= 0 || e.height <= 0) return splat(0);
    const int i = env_texel(e, env_uv(wi));
    const float* p = e.pixels + 3 * static_cast<size_t>(i);
    return make_f3(p[0], p[1], p[2]) * e.scale;
}

LUX_D float env_pdf_texel(const EnvLight& e, int index, float v) {
    if (!e.cdf || e.width <= 0 || e.height <= 0 || e.total <= 0) return 0;
    const int count = e.width * e.height;
    if (index < 0 || index >= count) return 0;
    float w = index == 0 ? e.cdf[0] : sub(e.cdf[index], e.cdf[index - 1]);
    if (w <= 0) return 0;
    float theta = mul(kPi, v);
    float sin_theta = fmaxf(1e-6f, sinf(theta));
    float uv_pdf = mul(w / e.total, static_cast<float>(count));
    return uv_pdf / mul(mul(mul(2.0f, kPi), kPi), sin_theta);
}

LUX_D float env_pdf(const EnvLight& e, f3 wi) {
    if (!e.pixels || !e.cdf || e.width <= 0 || e.height <= 0 || e.total <= 0) return 0;
    const float2 uv = env_uv(wi);
    return env_pdf_texel(e, env_texel(e, uv), uv.y);
}

// Texel by the running sums (the first texel whose sum reaches the target; a binary
// search finds the same texel as the reference's linear scan), then a uniform point in
// it.
LUX_D LightLi env_sample(const EnvLight& e, float select_u, float ux, float uy) {
    LightLi li;
    if (!e.pixels || !e.cdf || e.width <= 0 || e.height <= 0 || e.total <= 0) return li;
    const int count = e.width * e.height;
    const float target = mul(fminf(select_u, 0.99999994f), e.total);
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (target <= e.cdf[mid]) hi = mid;
        else lo = mid + 1;
    }
    const int index = target <= e.cdf[lo] ? lo : count - 1;
    const int x = index % e.width, y = index / e.width;
    const float u = add(static_cast<float>(x), ux) / static_cast<float>(e.width);
    const float v = add(static_cast<float>(y), uy) / static_cast<float>(e.height);
    const float phi = mul(mul(2.0f, kPi), u);
    const float theta = mul(kPi, v);
    const float st = sinf(theta);
    li.wi = make_f3(mul(cosf(phi), st), cosf(theta), mul(sinf(phi), st));
    li.distance = INFINITY;
    li.radiance = env_lookup(e, li.wi);
    li.pdf = env_pdf_texel(e, index, v);
    li.measure = kMeasureSolidAngle;
    li.valid = max_component(li.radiance) > 0 && li.pdf > 0;
    return li;
}

// ------------------------------------------------------------------ image emission
// image_asset_lookup_nearest (scene/scene_data.h:164-173): the texel under the wrapped
// texture coordinates, times scale.
LUX_D f3 image_lookup(const SceneView& sc, int image, float tu, float tv, f3 scale) {
    if (!sc.images || image < 0) return splat(0);
    const ImageView im = sc.images[image];
    if (!im.pixels || im.width <= 0 || im.height <= 0) return splat(0);
    const float u = sub(tu, floorf(tu));
    const float v = sub(tv, floorf(tv));
    const int x = static_cast<int>(fminf(static_cast<float>(im.width - 1), floorf(mul(u, static_cast<float>(im.width)))));
    const int y = static_cast<int>(fminf(static_cast<float>(im.height - 1), floorf(mul(v, static_cast<float>(im.height)))));
    const float* p = im.pixels + 3 * (static_cast<size_t>(y) * im.width + x);
    return make_f3(mul(p[0], scale.x), mul(p[1], scale.y), mul(p[2], scale.z));
}

// interpolate_triangle_uv (scene/scene_data.h:230-233) at barycentrics (u, v).
LUX_D void triangle_uv(const SceneTriShading& sh, float u, float v, float& tu, float& tv) {
    const float w = sub(sub(1.0f, u), v);
    tu = add(add(mul(w, sh.n0.w), mul(u, sh.n2.w)), mul(v, sh.uv.y));
    tv = add(add(mul(w, sh.n1.w), mul(u, sh.uv.x)), mul(v, sh.uv.z));
}

// gpu_diffuse_area_light_emission_value (gpu_scene_light_sampler.cuh:216-223).
LUX_D f3 area_light_emission(const SceneView& sc, const Light& L, int prim, float u, float v) {
    if (L.image < 0) return L.emission;
    float tu, tv;
    triangle_uv(sc.shading[prim], u, v, tu, tv);
    return image_lookup(sc, L.image, tu, tv, L.image_scale);
}

// sample_light_li (scene/scene_light_sampler.h:212-265 / gpu_scene_light_sampler.cuh:133-193).
LUX_D LightLi sample_light(const SceneView& sc, int sampler, f3 p, float select_u, float comp_u, float ux,
                           float uy) {
    LightLi li;
    float pmf;
    const int index = select_light(sc, sampler, p, select_u, pmf);
    if (index < 0 || !(pmf > 0)) return li;
    const Light L = sc.lights[index];
    if (L.kind == 0) {
        const SceneTri& t = sc.tris[L.primitive];
        f3 v0 = xyz(t.v0), v1 = xyz(t.v1), v2 = xyz(t.v2);
        f3 pos = sample_triangle_area(v0, v1, v2, ux, uy);
        f3 n = triangle_normal(v0, v1, v2);
        float pdf_area = L.area > 0 ? 1.0f / L.area : 0.0f;
        f3 to = pos - p;
        float d2 = length2(to);
        if (d2 <= mul(kRayEpsilon, kRayEpsilon)) return li;
        li.distance = sqrtf(d2);
        li.wi = vdiv(to, li.distance);
        li.position = pos;
        // sample_triangle_barycentric_uv (light/light_sampler.h:369-374) for the texel.
        const float s0 = sqrtf(ux);
        const f3 le = area_light_emission(sc, L, L.primitive, mul(s0, sub(1.0f, uy)), mul(s0, uy));
        li.radiance = eval_emission(le, L.two_sided, n, -li.wi);
        li.pdf = mul(pmf, solid_angle_pdf(pos, n, L.two_sided, pdf_area, p));
        li.measure = kMeasureSolidAngle;
        li.valid = max_component(li.radiance) > 0 && li.pdf > 0;
        return li;
    }
    if (L.kind == 1) {  // sample_point_light (light/light.h:161-175)
        f3 to = L.vec - p;
        float d2 = length2(to);
        if (d2 <= mul(kRayEpsilon, kRayEpsilon)) return li;
        li.distance = sqrtf(d2);
        li.wi = vdiv(to, li.distance);
        li.position = L.vec;
        li.radiance = vdiv(L.emission, d2);
        li.pdf = 1.0f;
        li.measure = kMeasureDiscrete;
        li.valid = max_component(li.radiance) > 0;
    } else if (L.kind == 2) {  // sample_distant_light (light/light.h:177-187)
        li.wi = normalize(L.vec);
        li.distance = INFINITY;
        li.radiance = L.emission;
        li.pdf = 1.0f;
        li.measure = kMeasureDiscrete;
        li.valid = max_component(li.radiance) > 0;
    } else if (L.kind == 4) {  // image infinite: the component draw picks the texel
        if (!sc.env || L.primitive < 0) return li;
        li = env_sample(sc.env[L.primitive], comp_u, ux, uy);
    } else {  // uniform infinite (light/light.h:144-150, 189-197)
        float z = sub(1.0f, mul(2.0f, ux));
        float r = sqrtf(fmaxf(0.0f, sub(1.0f, mul(z, z))));
        float phi = mul(mul(2.0f, kPi), uy);
        li.wi = make_f3(mul(r, cosf(phi)), z, mul(r, sinf(phi)));
        li.distance = INFINITY;
        li.radiance = L.emission;
        li.pdf = 1.0f / mul(4.0f, kPi);
        li.measure = kMeasureSolidAngle;
        li.valid = max_component(li.radiance) > 0;
    }
    li.pdf = mul(li.pdf, pmf);
    return li;
}

LUX_D f3 infinite_le(const SceneView& sc, f3 dir) {  // infinite_lights_le
    f3 le = splat(0);
    for (int i = 0; i < sc.light_count; ++i) {
        const Light& L = sc.lights[i];
        if (L.kind == 3) le = le + L.emission;
        else if (L.kind == 4 && sc.env && L.primitive >= 0) le = le + env_lookup(sc.env[L.primitive], dir);
    }
    return le;
}

LUX_D float infinite_pdf(const SceneView& sc, int sampler, f3 dir) {  // infinite_lights_pdf_li
    float pdf = 0;
    for (int i = 0; i < sc.light_count; ++i) {
        const Light& L = sc.lights[i];
        if (L.kind == 3) {
            pdf = add(pdf, mul(light_pmf(sc, sampler, splat(0.0f), i), 1.0f / mul(4.0f, kPi)));
        } else if (L.kind == 4 && sc.env && L.primitive >= 0) {
            pdf = add(pdf, mul(light_pmf(sc, sampler, splat(0.0f), i), env_pdf(sc.env[L.primitive], dir)));
        }
    }
    return pdf;
}

// ------------------------------------------------------------------ path state helpers

struct PathState {
    f3 thr;
    float eta;
    f3 prev_pos;
    float prev_pdf;
    int pixel, sample, depth, passthrough, measure;
    unsigned flags;
};

LUX_D PathState load_state(const PathPool& rt, int p) {
    PathState s;
    float4 a = rt.thr_eta[p];
    float4 b = rt.prev[p];
    int4 m = rt.meta[p];
    s.thr = xyz(a);
    s.eta = a.w;
    s.prev_pos = xyz(b);
    s.prev_pdf = b.w;
    s.pixel = m.x;
    s.sample = m.y;
    s.depth = m.z & 0xffff;
    s.passthrough = (m.z >> 16) & 0xffff;
    s.measure = m.w & 0xff;
    s.flags = static_cast<unsigned>(m.w) >> 8;
    return s;
}

LUX_D void store_state(const PathPool& rt, int p, const PathState& s) {
    rt.thr_eta[p] = make_float4(s.thr.x, s.thr.y, s.thr.z, s.eta);
    rt.prev[p] = make_float4(s.prev_pos.x, s.prev_pos.y, s.prev_pos.z, s.prev_pdf);
    rt.meta[p] = make_int4(s.pixel, s.sample, s.depth | (s.passthrough << 16),
                           s.measure | static_cast<int>(s.flags << 8));
}

LUX_D Pcg load_rng(const PathPool& rt, int p) {
    uint4 r = rt.rng[p];
    Pcg g;
    g.state = static_cast<uint64_t>(r.x) | (static_cast<uint64_t>(r.y) << 32);
    g.inc = static_cast<uint64_t>(r.z) | (static_cast<uint64_t>(r.w) << 32);
    return g;
}

LUX_D void store_rng(const PathPool& rt, int p, const Pcg& g) {
    rt.rng[p] = make_uint4(static_cast<unsigned>(g.state), static_cast<unsigned>(g.state >> 32),
                           static_cast<unsigned>(g.inc), static_cast<unsigned>(g.inc >> 32));
}

LUX_D void add_radiance(const PathPool& rt, int p, f3 v) {
    float4 r = rt.rad[p];
    rt.rad[p] = make_float4(add(r.x, v.x), add(r.y, v.y), add(r.z, v.z), 0.0f);
}

// Moves path p's state (everything but the per-bounce hit and shadow records) from pool
// src to slot q of pool dst.
LUX_D void copy_path(const PathPool& src, int p, const PathPool& dst, int q) {
    dst.thr_eta[q] = src.thr_eta[p];
    dst.rad[q] = src.rad[p];
    dst.prev[q] = src.prev[p];
    dst.meta[q] = src.meta[p];
    dst.rng[q] = src.rng[p];
    dst.ray_o[q] = src.ray_o[p];
    dst.ray_d[q] = src.ray_d[p];
}

LUX_D int material_of(const SceneView& sc, int prim) {
    return __float_as_int(__ldg(&sc.tris[prim].v0.w));
}

LUX_D int material_class(int type) {
    switch (type) {
        case kLambert: return 0;
        case kThinLambert: return 1;
        case kGgx: return 2;
        case kDielectric: return 3;
        default: return 4;
    }
}

// Emission seen at a hit (surface_light_le + area_light_pdf_solid_angle,
// scene/scene_light_sampler.h:318-465) at barycentrics (u, v).
LUX_D f3 surface_le(const SceneView& sc, int prim, const Material& m, f3 ng, f3 wo, float u,
                    float v) {
    int li = sc.primitive_light[prim];
    if (li >= 0 && li < sc.light_count && sc.lights[li].kind == 0) {
        const Light& L = sc.lights[li];
        return eval_emission(area_light_emission(sc, L, prim, u, v), L.two_sided, ng, wo);
    }
    if (m.emission_image >= 0) {  // gpu_eval_emission of an image-emissive material
        float tu, tv;
        triangle_uv(sc.shading[prim], u, v, tu, tv);
        return eval_emission(image_lookup(sc, m.emission_image, tu, tv, m.emission_scale),
                             m.two_sided, ng, wo);
    }
    if (max_component(m.emission) <= 0) return splat(0);
    return eval_emission(m.emission, m.two_sided, ng, wo);
}

LUX_D float surface_light_pdf(const SceneView& sc, int sampler, int prim, f3 ng, f3 pos,
                              f3 ref) {
    int li = sc.primitive_light[prim];
    if (li >= 0 && li < sc.light_count && sc.lights[li].kind == 0 && sc.lights[li].area > 0) {
        const Light& L = sc.lights[li];
        return mul(light_pmf(sc, sampler, ref, li), solid_angle_pdf(pos, ng, L.two_sided, 1.0f / L.area, ref));
    }
    return 0.0f;
}
// ------------------------------------------------------------------ per-path stages

struct CameraParams {
    int width, height;
    uint64_t seed;
    int frame_index, sample_offset;
};

// New camera path in slot p (generate_camera_rays_kernel; draw order jitter x, jitter y,
// lens 2D, time).
LUX_D void init_path(const PathPool& rt, const Camera& cam, int p, int pixel, int sample,
                     const CameraParams& c) {
    int x = pixel % c.width;
    int y = pixel / c.width;
    Pcg g = make_sampler(c.seed, c.frame_index, pixel, sample + c.sample_offset);
    float jx = g.next_float();
    float jy = g.next_float();
    float u = add(static_cast<float>(x), jx) / static_cast<float>(c.width);
    float v = add(static_cast<float>(c.height - 1 - y), jy) / static_cast<float>(c.height);
    float lx = g.next_float();
    float ly = g.next_float();
    (void)g.next_float();  // time
    f3 o, d;
    camera_ray(cam, u, v, lx, ly, o, d);
    PathState s;
    s.thr = splat(1.0f);
    s.eta = 1.0f;
    s.prev_pos = splat(0.0f);
    s.prev_pdf = 0.0f;
    s.pixel = pixel;
    s.sample = sample;
    s.depth = 0;
    s.passthrough = 0;
    s.measure = kMeasureNone;
    s.flags = 0;
    store_state(rt, p, s);
    store_rng(rt, p, g);
    rt.rad[p] = make_float4(0, 0, 0, 0);
    rt.ray_o[p] = make_float4(o.x, o.y, o.z, kRayEpsilon);
    rt.ray_d[p] = make_float4(d.x, d.y, d.z, INFINITY);
}

// Records the closest hit h of path p's ray: returns the material class of the hit, or
// -1 after adding the environment's radiance on a miss (cpu_path_tracer.cpp:415-428).
LUX_D int extend_finish(const PathPool& rt, const SceneView& sc, int sampler, int p,
                        const SceneHit& h) {
    if (h.prim >= 0) {
        rt.hit[p] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
        return material_class(sc.materials[material_of(sc, h.prim)].type);
    }
    const f3 dir = xyz(rt.ray_d[p]);
    f3 le = infinite_le(sc, dir);
    if (max_component(le) > 0) {
        PathState s = load_state(rt, p);
        if (s.depth == 0 || is_delta(s.flags)) {
            add_radiance(rt, p, s.thr * le);
        } else if (s.measure == kMeasureSolidAngle && s.prev_pdf > 0) {
            float w = power_heuristic(s.prev_pdf, infinite_pdf(sc, sampler, dir));
            add_radiance(rt, p, (s.thr * le) * w);
        }
    }
    return -1;
}

// Closest hit of path p's ray (one walk to completion), then extend_finish.
LUX_D int extend_path(const PathPool& rt, const SceneView& sc, int sampler, int p, int* error) {
    float4 a = rt.ray_o[p];
    float4 b = rt.ray_d[p];
    SceneHit h = scene_closest(sc, xyz(a), xyz(b), a.w, b.w, -1, error);
    return extend_finish(rt, sc, sampler, p, h);
}

// Closest hits of the paths in queue q[0, n) (q null: paths 0..n-1) by persistent warps:
// each lane advances its walk by at most `budget` steps per round, and lanes whose walk
// finished hand it to finish() and take the next path through one warp-aggregated
// atomic on *next_item, so lanes do not idle behind the longest walk of a static warp.
// tag_of(p) picks a path's scene once (view(tag) returns it); finish(p, hit) is called by
// every lane of the warp after each round in which some lane finished, with p = -1 for
// lanes that did not, so it may append to queues with warp-collective operations (and
// must do nothing for p = -1).
template <typename TagOf, typename View, typename Finish>
LUX_D void refill_walks(const PathPool& rt, const int* q, int n, int* next_item, int budget,
                        int* error, TagOf tag_of, View view, Finish finish) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    int p = -1;  // >= 0 active path, -1 needs one, -2 none left
    int tag = 0;
    TwoLevelWalk w;
    WalkStacks stacks;
    for (;;) {
        const bool need = p == -1;
        const unsigned m = __ballot_sync(0xffffffffu, need);
        if (m) {
            const int leader = __ffs(m) - 1;
            int base = 0;
            if (static_cast<int>(lane) == leader) base = atomicAdd(next_item, __popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                const int idx = base + __popc(m & lt);
                if (idx >= n) {
                    p = -2;
                } else {
                    p = q ? q[idx] : idx;
                    tag = tag_of(p);
                    const float4 a = rt.ray_o[p];
                    const float4 b = rt.ray_d[p];
                    w.init(view(tag), stacks, xyz(a), xyz(b), a.w, b.w, -1);
                }
            }
        }
        if (__all_sync(0xffffffffu, p == -2)) break;
        bool finished = false;
        if (p >= 0) {
            const SceneView& sc = view(tag);
            for (int s = 0; s < budget && !finished; ++s) finished = w.step(sc, stacks, error);
        }
        // finish() is warp-collective and does nothing for lanes that did not finish, so
        // a round in which no lane finished skips it.
        if (__any_sync(0xffffffffu, finished)) {
            SceneHit h = w.hit;
            if (h.prim < 0) h.t = INFINITY;
            finish(finished ? p : -1, tag, h);
        }
        if (finished) p = -1;
    }
}

// Shadow rays of the paths in queue q[0, n) by persistent warps with refilling lanes:
// each lane walks its ray's segments through pass-through surfaces exactly as
// shadow_path does (the same segment loop, one resumable walk per segment) and adds the
// NEE contribution when the ray is not blocked.  In a scene without pass-through
// materials the first hit already blocks the ray, and a hit exists exactly when a
// closest hit does, so the walk ends at the first accepted triangle.  deposit(p, value)
// adds the contribution to wherever path p's radiance lives.
template <typename TagOf, typename View, typename Deposit>
LUX_D void refill_shadows(const PathPool& rt, const int* q, int n, int* next_item, int budget,
                          int* error, TagOf tag_of, View view, Deposit deposit,
                          unsigned long long& segments) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    int p = -1;  // >= 0 active path, -1 needs one, -2 none left
    int tag = 0, seg = 0;
    f3 o, d, tr;
    float tmax = 0;
    TwoLevelWalk w;
    WalkStacks stacks;
    for (;;) {
        const bool need = p == -1;
        const unsigned m = __ballot_sync(0xffffffffu, need);
        if (m) {
            const int leader = __ffs(m) - 1;
            int base = 0;
            if (static_cast<int>(lane) == leader) base = atomicAdd(next_item, __popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                const int idx = base + __popc(m & lt);
                if (idx >= n) {
                    p = -2;
                } else {
                    p = q[idx];
                    tag = tag_of(p);
                    const float4 a = rt.sh_o[p];
                    const float4 b = rt.sh_d[p];
                    o = xyz(a);
                    d = xyz(b);
                    tmax = a.w;
                    tr = splat(1.0f);
                    seg = 0;
                    ++segments;
                    const SceneView& sv = view(tag);
                    w.init(sv, stacks, o, d, kRayEpsilon, tmax, __float_as_int(b.w),
                           !sv.has_passthrough);
                }
            }
        }
        if (__all_sync(0xffffffffu, p == -2)) break;
        if (p < 0) continue;
        const SceneView& sc = view(tag);
        for (int s = 0; s < budget; ++s) {
            if (!w.step(sc, stacks, error)) continue;
            bool end = false, blocked = false;
            const SceneHit& h = w.hit;
            if (h.prim < 0) {
                end = true;
            } else {
                const Material mat = sc.materials[material_of(sc, h.prim)];
                if (!is_passthrough(mat)) {
                    blocked = true;
                    end = true;
                } else {
                    tr = tr * passthrough_transmittance(mat);
                    const float adv = add(h.t, kRayEpsilon);
                    if (max_component(tr) <= 0 || adv >= tmax) {
                        end = true;
                    } else if (++seg >= kShadowSegments) {
                        atomicOr(error, kErrLoopBound);
                        blocked = true;
                        end = true;
                    } else {
                        o = o + d * adv;
                        tmax = sub(tmax, adv);
                        ++segments;
                        w.init(sc, stacks, o, d, kRayEpsilon, tmax, -1);
                    }
                }
            }
            if (end) {
                if (!blocked && max_component(tr) > 0) {
                    const float4 c = rt.sh_c[p], t = rt.sh_t[p];
                    deposit(p, xyz(t) * ((xyz(c) * tr) * c.w));
                }
                p = -1;
                break;
            }
        }
    }
}

struct ShadeOut {
    bool spawn = false;   // ray_o/ray_d[p] hold the next ray
    bool shadow = false;  // sh_*[p] hold a shadow ray
};

// ------------------------------------------------------------------ debug images
// The reference wavefront tracer's debug images (integrator/wavefront_debug.cuh,
// wavefront_kernels.cu:287-305, 475-482, 586-592), per-pixel sums over samples:
//   ng / ns   at the camera ray's hit: 0.5 * (normalize(n) + 1) of the geometric normal /
//             of the shading normal turned to the geometric side; nothing on a miss;
//   shadow    at the path's first scattering hit (depth 0, after pass-through surfaces),
//             when it samples a light: orange (1, 0.5, 0) when the light sample is
//             invalid, purple (0.5, 0, 1) when the unoccluded estimate is, else the
//             classification of its shadow ray (shadow_aov_color).
//   path log  (on when log_count is set) one lux_path_log_record per surface vertex a
//             path reaches (integrator/pathstate.cuh:41-96), at an atomically taken
//             index; the index keeps counting past capacity so the host learns the size
//             needed.
struct DebugTargets {
    float* shadow = nullptr;
    float* ng = nullptr;
    float* ns = nullptr;
    lux_path_log_record* log = nullptr;
    unsigned long long* log_count = nullptr;
    long long log_capacity = 0;
    int sample_offset = 0;
    // Traversal totals (box tests, triangle tests, instance visits) of every extension
    // and shadow walk, or null.
    unsigned long long* walk_counts = nullptr;
};

// What the shading of one vertex decided, for its path log record
// (SurfaceStageLogState, integrator/wavefront_kernels.cu:140-151).
struct VertexLog {
    f3 wi = make_f3(0, 0, 0);
    float bsdf_pdf = 0, light_pdf = 0;
    int bsdf_measure = kMeasureNone, light_measure = kMeasureNone, source = 0;
    unsigned bsdf_flags = 0;
    unsigned events = LUX_PATH_EVENT_SURFACE_HIT;
};

constexpr int kSourceBsdf = 2;  // SampleSource::BSDF

// record_surface_vertex / record_path_vertex (integrator/wavefront_kernels.cu:84-138,
// integrator/pathstate.cuh:82-96) for the vertex at hit prim of path state s.
LUX_D void log_vertex(const DebugTargets& dbg, const SceneView& sc, const PathState& s,
                      int vertex, int depth, int prim, f3 pos, f3 ng, f3 ns, f3 wo, f3 thr_before,
                      f3 thr_after, const VertexLog& v, unsigned termination) {
    if (!dbg.log_count) return;
    const unsigned long long index = atomicAdd(dbg.log_count, 1ull);
    if (index >= static_cast<unsigned long long>(dbg.log_capacity)) return;
    const SceneTri tri = sc.tris[prim];
    lux_path_log_record r;
    r.pixel_index = s.pixel;
    r.sample_index = dbg.sample_offset + s.sample;
    r.depth = depth;
    r.triangle_id = prim;
    r.instance_id = __float_as_int(tri.v1.w);
    r.mesh_id = sc.instances[r.instance_id].blas;
    r.local_primitive_id = __float_as_int(tri.v2.w);
    r.primitive_kind = 1;
    r.material_id = __float_as_int(tri.v0.w);
    r.vertex = vertex;
    const f3 vecs[7] = {pos, ng, ns, wo, v.wi, thr_before, thr_after};
    float* dst[7] = {r.position, r.ng, r.ns, r.wo, r.wi, r.throughput_before, r.throughput_after};
    for (int k = 0; k < 7; ++k) {
        dst[k][0] = vecs[k].x;
        dst[k][1] = vecs[k].y;
        dst[k][2] = vecs[k].z;
    }
    r.bsdf_pdf = v.bsdf_pdf;
    r.guide_pdf = 0.0f;
    r.light_pdf = v.light_pdf;
    r.bsdf_pdf_measure = static_cast<uint8_t>(v.bsdf_measure);
    r.guide_pdf_measure = 0;
    r.light_pdf_measure = static_cast<uint8_t>(v.light_measure);
    r.sample_source = static_cast<uint8_t>(v.source);
    r.bsdf_flags = v.bsdf_flags;
    r.termination_flags = termination;
    r.event_flags = v.events | (termination ? LUX_PATH_EVENT_TERMINATED : 0u);
    dbg.log[index] = r;
}

LUX_D void aov_add(float* image, int pixel, f3 c) {
    atomicAdd(image + 3 * size_t(pixel), c.x);
    atomicAdd(image + 3 * size_t(pixel) + 1, c.y);
    atomicAdd(image + 3 * size_t(pixel) + 2, c.z);
}

LUX_D f3 encode_normal_color(f3 n) { return (normalize(n) + splat(1.0f)) * 0.5f; }

// primary_normal_debug_color for the camera ray's closest hit h of path p.
LUX_D void aov_primary(const PathPool& rt, const SceneView& sc, int p, const SceneHit& h,
                       const DebugTargets& aov) {
    const int4 meta = rt.meta[p];
    if (meta.z != 0 || h.prim < 0) return;  // depth and pass-through count both zero
    const SceneTri tri = sc.tris[h.prim];
    const f3 ng = triangle_normal(xyz(tri.v0), xyz(tri.v1), xyz(tri.v2));
    if (aov.ng) aov_add(aov.ng, meta.x, encode_normal_color(ng));
    if (aov.ns) {
        f3 ns = shading_normal(sc.shading[h.prim], ng, h.u, h.v);
        if (dot(ng, ns) < 0) ns = -ns;
        aov_add(aov.ns, meta.x, encode_normal_color(ns));
    }
}

// shadow_debug_classification_color: red when the shading normal faces the light but
// the geometric normal does not; unblocked: blue-ish after pass-through surfaces, else
// dark grey; blocked by the source's own material within 16 epsilon: yellow; by a back
// face of it: blue (magenta near a mesh boundary edge, which these scenes do not carry);
// by a front face of it: cyan; by another material: green.
LUX_D f3 shadow_aov_color(const SceneView& sc, int source_prim, f3 ng, f3 ns, f3 dir,
                          int occluder, float hit_t, int passthrough_hits) {
    const float shading_cos = dot(ns, dir);
    const float geometric_cos = dot(ng, dir);
    if (shading_cos > 0 && geometric_cos <= 0) return make_f3(1, 0, 0);
    if (occluder < 0) return passthrough_hits > 0 ? make_f3(0, 0.35f, 0.8f) : splat(0.03f);
    const bool same = material_of(sc, occluder) == material_of(sc, source_prim);
    if (same && hit_t < mul(16.0f, kRayEpsilon)) return make_f3(1, 1, 0);
    if (same) {
        const SceneTri o = sc.tris[occluder];
        const bool back = dot(triangle_normal(xyz(o.v0), xyz(o.v1), xyz(o.v2)), -dir) <= 0;
        return back ? make_f3(0, 0, 1) : make_f3(0, 1, 1);
    }
    return make_f3(0, 1, 0);
}

// Shading of the hit stored for path p (cpu_path_tracer.cpp:430-497).  With kAov, also
// the shadow debug image's light-sample verdict at depth 0, shadow rays at depth 0 are
// marked (sh_t.w = 1) for classification, and the vertex goes to the path log at each
// exit evaluate_hit_kernel records one (integrator/wavefront_kernels.cu:397-555).
template <bool kAov = false>
LUX_D ShadeOut shade_path(const PathPool& rt, const SceneView& sc, int sampler, int max_depth,
                          int p, const DebugTargets& aov = DebugTargets{}) {
    ShadeOut out;
    float4 ra = rt.ray_o[p], rb = rt.ray_d[p], hh = rt.hit[p];
    f3 ro = xyz(ra), rd = xyz(rb);
    int prim = __float_as_int(hh.w);
    float t = hh.x, hu = hh.y, hv = hh.z;
    const SceneTri tri = sc.tris[prim];
    f3 v0 = xyz(tri.v0), v1 = xyz(tri.v1), v2 = xyz(tri.v2);
    const Material m = sc.materials[__float_as_int(tri.v0.w)];
    PathState s = load_state(rt, p);
    const int step = s.depth + s.passthrough;
    f3 pos = ro + rd * t;                    // Ray::at
    f3 ng = triangle_normal(v0, v1, v2);
    f3 wo = -rd;
    const bool logging = kAov && aov.log_count != nullptr;
    const f3 thr0 = s.thr;
    VertexLog vl;
    // Logs this vertex with throughput_after thr1 and the given termination.
    auto log = [&](f3 thr1, unsigned termination) {
        if (!logging) return;
        f3 n = shading_normal(sc.shading[prim], ng, hu, hv);
        if (dot(ng, n) < 0) n = -n;
        log_vertex(aov, sc, s, step, s.depth, prim, pos, ng, n, wo, thr0, thr1, vl, termination);
    };
    // Emission with MIS (cpu_path_tracer.cpp:434-447).
    f3 le = surface_le(sc, prim, m, ng, wo, hu, hv);
    if (max_component(le) > 0) {
        if (s.depth == 0 || is_delta(s.flags)) {
            add_radiance(rt, p, s.thr * le);
            vl.events |= LUX_PATH_EVENT_EMISSION;
        } else if (s.measure == kMeasureSolidAngle && s.prev_pdf > 0) {
            float lpdf = surface_light_pdf(sc, sampler, prim, ng, pos, s.prev_pos);
            add_radiance(rt, p, (s.thr * le) * power_heuristic(s.prev_pdf, lpdf));
            vl.events |= LUX_PATH_EVENT_EMISSION;
        }
    }
    if (is_passthrough(m)) {  // cpu_path_tracer.cpp:449-455
        s.thr = s.thr * passthrough_transmittance(m);
        vl.events |= LUX_PATH_EVENT_PASSTHROUGH | LUX_PATH_EVENT_DELTA;
        vl.wi = normalize(-wo);
        vl.bsdf_pdf = 1.0f;
        vl.bsdf_measure = kMeasureDiscrete;
        vl.source = kSourceBsdf;
        vl.bsdf_flags = kFlagDeltaTransmission | kFlagTransmission;
        if (max_component(s.thr) > 0 && step < max_depth) {
            vl.events |= LUX_PATH_EVENT_SPAWNED_RAY;
            log(s.thr, 0);
            s.passthrough += 1;
            f3 no = pos + rd * kRayEpsilon;
            rt.ray_o[p] = make_float4(no.x, no.y, no.z, kRayEpsilon);
            rt.ray_d[p] = make_float4(rd.x, rd.y, rd.z, INFINITY);
            out.spawn = true;
        } else {
            log(s.thr, max_component(s.thr) <= 0 ? LUX_PATH_END_ZERO_THROUGHPUT
                                                 : LUX_PATH_END_MAX_DEPTH);
        }
        store_state(rt, p, s);
        return out;
    }
    if (!is_scattering(m)) {
        log(thr0, LUX_PATH_END_NON_SCATTERING);
        return out;
    }
    if (step >= max_depth || s.depth >= max_depth) {
        log(thr0, LUX_PATH_END_MAX_DEPTH);
        return out;
    }
    SceneTriShading sh = sc.shading[prim];
    f3 ns = shading_normal(sh, ng, hu, hv);
    if (dot(ng, ns) < 0) ns = -ns;   // make_surface_interaction
    Interaction it{pos, ng, ns, wo};
    Pcg g = load_rng(rt, p);
    if (has_direct_lighting_lobe(m)) {  // estimate_direct_light, :122-158
        float su = g.next_float();
        float cu = g.next_float();
        float lx = g.next_float();
        float ly = g.next_float();
        LightLi li = sample_light(sc, sampler, pos, su, cu, lx, ly);
        int verdict = 0;  // 0 light sample invalid, 1 estimate invalid, 2 valid
        if (li.valid) vl.events |= LUX_PATH_EVENT_DIRECT_LIGHT_SAMPLED;
        if (li.valid && li.pdf > 0) {
            verdict = 1;
            vl.light_pdf = li.pdf;  // pdf_light_solid_angle, logged as a solid angle
            vl.light_measure = kMeasureSolidAngle;
            f3 f = eval_bsdf(m, it, li.wi);
            float cs = abs_cosine(ns, li.wi);
            float pb = pdf_bsdf(m, it, li.wi);
            if (max_component(f) > 0 && max_component(li.radiance) > 0 && cs > 0) {
                verdict = 2;
                vl.events |= LUX_PATH_EVENT_DIRECT_LIGHT_VALID;
                f3 contrib = (f * li.radiance) * (cs / li.pdf);
                float mis = li.measure == kMeasureDiscrete ? 1.0f : power_heuristic(li.pdf, pb);
                f3 off = dot(li.wi, ng) >= 0 ? ng : -ng;
                f3 so = pos + off * kRayEpsilon;
                f3 sd = li.wi;
                float smax = INFINITY;
                bool ok = true;
                if (li.distance < INFINITY) {  // trace_shadow(from, to)
                    f3 to = li.position - so;
                    float dist = length(to);
                    if (dist <= kRayEpsilon) {
                        ok = false;
                    } else {
                        sd = vdiv(to, dist);
                        smax = sub(dist, kRayEpsilon);
                    }
                }
                const bool mark = kAov && aov.shadow && s.depth == 0 && sc.light_count > 0 &&
                                  sc.total_light_power > 0;
                if (!ok && mark) {  // make_shadow_work_item_li: a zero-length ray, no light
                    sd = li.wi;
                    smax = kRayEpsilon;
                    contrib = splat(0.0f);
                    ok = true;
                }
                if (ok) {
                    out.shadow = true;
                    rt.sh_o[p] = make_float4(so.x, so.y, so.z, smax);
                    rt.sh_d[p] = make_float4(sd.x, sd.y, sd.z, __int_as_float(prim));
                    rt.sh_c[p] = make_float4(contrib.x, contrib.y, contrib.z, mis);
                    rt.sh_t[p] = make_float4(s.thr.x, s.thr.y, s.thr.z, mark ? 1.0f : 0.0f);
                }
            }
        }
        if (kAov && aov.shadow && s.depth == 0 && verdict < 2 && sc.light_count > 0 &&
            sc.total_light_power > 0)
            aov_add(aov.shadow, s.pixel, verdict == 0 ? make_f3(1, 0.5f, 0) : make_f3(0.5f, 0, 1));
    }
    float bx = g.next_float();
    float by = g.next_float();
    BsdfSample bs = sample_bsdf(m, it, bx, by);
    vl.wi = bs.wi;
    vl.bsdf_flags = bs.flags;
    vl.events |= LUX_PATH_EVENT_BSDF_SAMPLED | (is_delta(bs.flags) ? LUX_PATH_EVENT_DELTA : 0u);
    if (bs.pdf > 0) {
        vl.bsdf_pdf = bs.pdf;
        vl.bsdf_measure = bs.measure;
    }
    if (!(bs.pdf > 0 && max_component(bs.weight) > 0)) log(thr0, LUX_PATH_END_INVALID_BSDF);
    if (bs.pdf > 0 && max_component(bs.weight) > 0) {
        f3 nthr = s.thr * bs.weight;
        float neta = mul(s.eta, is_transmission(bs.flags) && bs.eta > 0 ? mul(bs.eta, bs.eta) : 1.0f);
        bool alive = true;
        vl.source = kSourceBsdf;
        if (s.depth > 2) {  // path_transport.cuh:58-84
            float prob = fminf(0.95f, mul(max_component(nthr), neta));
            float ru = g.next_float();
            if (ru <= prob) nthr = vdiv(nthr, prob);
            else alive = false;
        }
        if (!alive) log(nthr, LUX_PATH_END_RUSSIAN_ROULETTE);
        if (alive) {
            vl.events |= LUX_PATH_EVENT_SPAWNED_RAY;
            log(nthr, 0);
            s.thr = nthr;
            s.eta = neta;
            s.prev_pdf = bs.pdf;
            s.measure = bs.measure;
            s.flags = bs.flags;
            s.prev_pos = pos;
            s.depth += 1;
            f3 off = dot(bs.wi, ng) >= 0 ? ng : -ng;   // spawn_scatter_ray
            f3 no = pos + off * kRayEpsilon;
            rt.ray_o[p] = make_float4(no.x, no.y, no.z, kRayEpsilon);
            rt.ray_d[p] = make_float4(bs.wi.x, bs.wi.y, bs.wi.z, INFINITY);
            out.spawn = true;
        }
    }
    store_state(rt, p, s);
    store_rng(rt, p, g);
    return out;
}

// Shadow ray of path p through pass-through surfaces (trace_shadow,
// cpu_path_tracer.cpp:27-73); adds throughput * ((contribution * T) * mis).  With kAov,
// a ray marked at shading adds its classification colour to the shadow debug image.
template <bool kAov = false>
LUX_D void shadow_path(const PathPool& rt, const SceneView& sc, int p, int* error,
                       unsigned long long& segments, const DebugTargets& aov = DebugTargets{}) {
    float4 a = rt.sh_o[p], b = rt.sh_d[p];
    f3 o = xyz(a), d = xyz(b);
    float tmax = a.w;
    float tmin = kRayEpsilon;
    int ignored = __float_as_int(b.w);
    f3 tr = splat(1.0f);
    bool blocked = false;
    int occluder = -1, crossed = 0;
    float occluder_t = 0;
    for (int seg = 0;; ++seg) {
        if (seg >= kShadowSegments) {
            atomicOr(error, kErrLoopBound);
            blocked = true;
            break;
        }
        ++segments;
        SceneHit h;
        if (kAov && aov.walk_counts) {
            WalkCounts wc;
            h = scene_closest<true>(sc, o, d, tmin, tmax, ignored, error, &wc);
            atomicAdd(aov.walk_counts, wc.boxes);
            atomicAdd(aov.walk_counts + 1, wc.tris);
            atomicAdd(aov.walk_counts + 2, wc.instances);
        } else {
            h = scene_closest(sc, o, d, tmin, tmax, ignored, error);
        }
        if (h.prim < 0) break;
        const Material m = sc.materials[material_of(sc, h.prim)];
        if (!is_passthrough(m)) {
            blocked = true;
            occluder = h.prim;
            occluder_t = h.t;
            break;
        }
        ++crossed;
        tr = tr * passthrough_transmittance(m);
        if (max_component(tr) <= 0) break;
        float adv = add(h.t, kRayEpsilon);
        if (adv >= tmax) break;
        o = o + d * adv;
        tmax = sub(tmax, adv);
        tmin = kRayEpsilon;
        ignored = -1;
    }
    if (!blocked && max_component(tr) > 0) {
        float4 c = rt.sh_c[p], t = rt.sh_t[p];
        f3 contrib = (xyz(c) * tr) * c.w;
        add_radiance(rt, p, xyz(t) * contrib);
    }
    if (kAov && aov.shadow && rt.sh_t[p].w == 1.0f) {
        const int source = __float_as_int(rt.sh_d[p].w);
        const SceneTri tri = sc.tris[source];
        const f3 ng = triangle_normal(xyz(tri.v0), xyz(tri.v1), xyz(tri.v2));
        const float4 hh = rt.hit[p];
        f3 ns = shading_normal(sc.shading[source], ng, hh.y, hh.z);
        if (dot(ng, ns) < 0) ns = -ns;
        aov_add(aov.shadow, rt.meta[p].x,
                shadow_aov_color(sc, source, ng, ns, d, occluder, occluder_t, crossed));
    }
}

LUX_D void warp_add(unsigned long long* counter, unsigned long long v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(counter, v);
}

}  // namespace
}  // namespace pt
}  // namespace lux
