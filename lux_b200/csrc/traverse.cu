// Ray traversal (closest hit, any hit) and box-overlap queries over the LBVH.
//
// Closest hit reproduces the reference's stackless walk (bvh/bvh_device.cuh:43-90)
// decision for decision, at half the node fetches:
//   * nodes are visited left child first, so the visit order is the reference's
//     preorder and equal-t ties keep the first triangle found;
//   * both child boxes are tested when their parent is fetched; a right child that is
//     deferred keeps its slab entry distance tn, and when popped it is skipped iff
//     tn > best_t, which is exactly the reference's slab verdict for that node under
//     the t_max current at its visit (its t_max-free part was already checked);
//   * triangles pass iff t_min < t < best_t (strict, as geometry/triangle.h:51).
// Overlap queries follow bvh/bvh_overlap.cu:25-184 (self pairs a < b; cross pairs
// (left, right)), with warp-aggregated appends instead of a block-wide staging loop.

#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/lux_gpu.h"
#include "lux_internal.h"
#include "lux_wide.cuh"

namespace lux {
namespace {

constexpr int kTraceThreads = 128;
#ifndef LUX_TRACE_BLOCKS
#define LUX_TRACE_BLOCKS 10
#endif
constexpr int kTraceBlocks = LUX_TRACE_BLOCKS;   // resident blocks per SM of the wide walk
constexpr int kStack = 96;  // > max Karras depth: 64 (30-bit keys) or 95 (63-bit + index)

struct RayHit {
    int k;      // sorted leaf index of the best hit, -1 none
    float t;
};

LUX_D ray3 load_ray(const float4* rays, int i) {
    float4 a = __ldg(rays + 2 * i);
    float4 b = __ldg(rays + 2 * i + 1);
    return ray3{make_f3(a.x, a.y, a.z), a.w, make_f3(b.x, b.y, b.z), b.w};
}

struct TraceCounts {
    unsigned boxes = 0;
    unsigned tris = 0;
};

template <bool AnyHit, bool Count = false>
LUX_D RayHit trace_one(const BvhView& bvh, const ray3& ray, int* error,
                       TraceCounts* counts = nullptr) {
    RayHit best{-1, ray.tmax};
    if (bvh.n <= 0) return best;
    slab_ray sr = make_slab_ray(ray);
    float tn;
    if (Count) counts->boxes += 1;
    if (!slab_hit(sr, load_root(bvh.root), best.t, tn)) return best;

    int stack_h[kStack];
    float stack_t[kStack];
    int sp = 0;
    int cur = bvh.n == 1 ? ~0 : 0;
    // A tree visit touches each node at most once: 2n steps bound any correct walk.
    const long long bound = 2ll * bvh.n + 64;
    for (long long step = 0;; ++step) {
        if (step > bound || cur >= bvh.n - 1 || ~cur >= bvh.n) {
            atomicOr(error, kErrLoopBound);
            return RayHit{-1, ray.tmax};
        }
        if (cur >= 0) {
            BvhNode nd = load_node(bvh.nodes, cur);
            float tl, tr;
            if (Count) counts->boxes += 2;
            bool hl = slab_hit(sr, node_left_box(nd), best.t, tl);
            bool hr = slab_hit(sr, node_right_box(nd), best.t, tr);
            if (hl) {
                if (hr) {
                    if (sp < kStack) {
                        stack_h[sp] = nd.ch.y;
                        stack_t[sp] = tr;
                        ++sp;
                    } else {
                        atomicOr(error, kErrStackOverflow);
                        return RayHit{-1, ray.tmax};
                    }
                }
                cur = nd.ch.x;
                continue;
            }
            if (hr) {
                cur = nd.ch.y;
                continue;
            }
        } else {
            int k = ~cur;
            const float4* tp = reinterpret_cast<const float4*>(bvh.tris + k);
            float4 p0 = __ldg(tp);
            float4 p1 = __ldg(tp + 1);
            float4 p2 = __ldg(tp + 2);
            float t, u, v;
            if (Count) counts->tris += 1;
            if (moller_trumbore(ray.o, ray.d, make_f3(p0.x, p0.y, p0.z),
                                make_f3(p1.x, p1.y, p1.z), make_f3(p2.x, p2.y, p2.z), t, u, v)
                && t > ray.tmin && t < best.t) {
                best.k = k;
                best.t = t;
                if (AnyHit) return best;
            }
        }
        // Pop the next deferred right child that still passes under the current best.
        bool resumed = false;
        while (sp > 0) {
            --sp;
            if (!(stack_t[sp] > best.t)) {
                cur = stack_h[sp];
                resumed = true;
                break;
            }
        }
        if (!resumed) break;
    }
    return best;
}

template <bool AnyHit>
__global__ void __launch_bounds__(kTraceThreads) k_trace(BvhView bvh, const float4* rays,
                                                         int nrays, int* hit_id, float* hit_t,
                                                         int* error) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrays) return;
    ray3 ray = load_ray(rays, i);
    RayHit h = trace_one<AnyHit>(bvh, ray, error);
    int id = -1;
    if (h.k >= 0) id = __float_as_int(__ldg(reinterpret_cast<const float*>(bvh.tris + h.k) + 3));
    hit_id[i] = id;
    if (hit_t) hit_t[i] = h.k >= 0 ? h.t : INFINITY;
}

// One ray per thread over the 4-wide nodes (lux_wide.cuh): the same verdicts as
// trace_one with half the dependent node fetches.
template <bool AnyHit>
__global__ void __launch_bounds__(kTraceThreads) k_trace_wide(BvhView bvh, const float4* rays,
                                                              int nrays, int* hit_id,
                                                              float* hit_t, int* error) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrays) return;
    const ray3 ray = load_ray(rays, i);
    const slab_ray sr = make_slab_ray(ray);
    float best_t = ray.tmax;
    int best_k = -1;
    bool ok = wide_walk(bvh, sr, best_t, error,
                        [&](int k, const float4& p0, const float4& p1, const float4& p2,
                            float& bt) -> bool {
        float t, u, v;
        if (moller_trumbore(ray.o, ray.d, make_f3(p0.x, p0.y, p0.z), make_f3(p1.x, p1.y, p1.z),
                            make_f3(p2.x, p2.y, p2.z), t, u, v)
            && t > ray.tmin && t < bt) {
            best_k = k;
            bt = t;
            return AnyHit;
        }
        return false;
    });
    if (!ok) best_k = -1;
    int id = -1;
    if (best_k >= 0) id = __float_as_int(__ldg(reinterpret_cast<const float*>(bvh.tris + best_k) + 3));
    hit_id[i] = id;
    if (hit_t) hit_t[i] = best_k >= 0 ? best_t : INFINITY;
}

// Persistent traversal: each warp keeps 32 rays in flight and advances each by at most
// `budget` steps per round; lanes whose ray finished fetch the next ray index with one
// warp-aggregated atomic, so lanes do not idle until the longest ray of a static warp
// finishes.  A step is one node fetch (two child boxes) or one triangle test followed by
// the pops it enables.  Decisions are those of trace_one, step for step.
LUX_D unsigned lanemask_lt_u() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <bool AnyHit>
__global__ void __launch_bounds__(kTraceThreads) k_trace_persistent(
        BvhView bvh, const float4* rays, int nrays, int* hit_id, float* hit_t,
        unsigned* ray_counter, int budget, int* error) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt_u();
    const box3 root = load_root(bvh.root);
    const unsigned bound = 2u * static_cast<unsigned>(bvh.n) + 64u;  // n <= 2^30

    int ray_idx = -1;   // >= 0 active ray, -1 needs a ray, -2 no rays left
    ray3 ray;
    slab_ray sr;
    octant_ray orr;
    bool fast = true;
    float best_t = 0.0f;
    int best_k = -1;
    int cur = 0;
    int sp = 0;
    unsigned steps = 0;
    bool root_missed = false;
    int stack_h[kStack];
    float stack_t[kStack];

    for (;;) {
        // Refill finished lanes (one atomic per warp).
        bool need = ray_idx == -1;
        unsigned need_mask = __ballot_sync(0xffffffffu, need);
        if (need_mask) {
            int leader = __ffs(need_mask) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(ray_counter, __popc(need_mask));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                unsigned idx = base + __popc(need_mask & lt);
                if (idx >= static_cast<unsigned>(nrays)) {
                    ray_idx = -2;
                } else {
                    ray_idx = static_cast<int>(idx);
                    ray = load_ray(rays, ray_idx);
                    sr = make_slab_ray(ray);
                    fast = sr.parallel == 0;
                    orr = make_octant_ray(sr);
                    best_t = ray.tmax;
                    best_k = -1;
                    sp = 0;
                    steps = 0;
                    float tn;
                    root_missed = bvh.n <= 0 || !slab_hit(sr, root, best_t, tn);
                    cur = bvh.n == 1 ? ~0 : 0;
                }
            }
        }
        if (__all_sync(0xffffffffu, ray_idx == -2)) break;

        bool done = false;
        if (ray_idx >= 0) {
            if (root_missed) done = true;
            for (int s = 0; s < budget && !done; ++s) {
                if (++steps > bound || cur >= bvh.n - 1 || ~cur >= bvh.n) {
                    atomicOr(error, kErrLoopBound);
                    best_k = -1;
                    best_t = ray.tmax;
                    done = true;
                    break;
                }
                bool pop = true;
                if (cur >= 0) {
                    BvhNode nd = load_node(bvh.nodes, cur);
                    float tl, tr;
                    bool hl, hr;
                    if (fast) {
                        hl = octant_hit(orr, node_left_box(nd), best_t, tl);
                        hr = octant_hit(orr, node_right_box(nd), best_t, tr);
                    } else {
                        hl = slab_hit(sr, node_left_box(nd), best_t, tl);
                        hr = slab_hit(sr, node_right_box(nd), best_t, tr);
                    }
                    if (hl) {
                        if (hr) {
                            if (sp >= kStack) {
                                atomicOr(error, kErrStackOverflow);
                                best_k = -1;
                                best_t = ray.tmax;
                                done = true;
                                break;
                            }
                            stack_h[sp] = nd.ch.y;
                            stack_t[sp] = tr;
                            ++sp;
                        }
                        cur = nd.ch.x;
                        pop = false;
                    } else if (hr) {
                        cur = nd.ch.y;
                        pop = false;
                    }
                } else {
                    int k = ~cur;
                    const float4* tp = reinterpret_cast<const float4*>(bvh.tris + k);
                    float4 p0 = __ldg(tp);
                    float4 p1 = __ldg(tp + 1);
                    float4 p2 = __ldg(tp + 2);
                    float t, u, v;
                    if (moller_trumbore(ray.o, ray.d, make_f3(p0.x, p0.y, p0.z),
                                        make_f3(p1.x, p1.y, p1.z), make_f3(p2.x, p2.y, p2.z),
                                        t, u, v)
                        && t > ray.tmin && t < best_t) {
                        best_k = k;
                        best_t = t;
                        if (AnyHit) {
                            done = true;
                            break;
                        }
                    }
                }
                if (pop) {
                    bool resumed = false;
                    while (sp > 0) {
                        --sp;
                        if (!(stack_t[sp] > best_t)) {
                            cur = stack_h[sp];
                            resumed = true;
                            break;
                        }
                    }
                    if (!resumed) done = true;
                }
            }
        }
        if (done) {
            int id = -1;
            if (best_k >= 0)
                id = __float_as_int(__ldg(reinterpret_cast<const float*>(bvh.tris + best_k) + 3));
            hit_id[ray_idx] = id;
            if (hit_t) hit_t[ray_idx] = best_k >= 0 ? best_t : INFINITY;
            ray_idx = -1;
        }
    }
}

// Persistent warps with refill (as k_trace_persistent) over the 4-wide nodes: a step is
// one wide-node fetch (four child boxes) or one triangle test, followed by the pops it
// enables.  Decisions are those of wide_walk, step for step.
// 10 resident blocks per SM (at most 48 registers): occupancy hides the node-load
// latency that bounds this kernel.  The cap spills 44 bytes per thread, and the extra
// warps still win: 468 against 439 Mrays/s at 64 registers and 425 at 40 (1,048,576
// triangles, 4,194,304 rays, B200).  The deferred-child stack lives in local memory and
// its reads mostly miss L1; keeping an entry's node and entry distance in one 8-byte
// record (one access per push or pop rather than two) gives 479 against 467 Mrays/s.
template <bool AnyHit>
__global__ void __launch_bounds__(kTraceThreads, kTraceBlocks) k_trace_wide_persistent(
        BvhView bvh, const float4* rays, int nrays, int* hit_id, float* hit_t,
        unsigned* ray_counter, int budget, int* error) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt_u();
    const box3 root = load_root(bvh.root);
    const unsigned bound = 2u * static_cast<unsigned>(bvh.n) + 64u;  // n <= 2^30

    int ray_idx = -1;   // >= 0 active ray, -1 needs a ray, -2 no rays left
    ray3 ray;
    slab_ray sr;
    octant_ray orr;
    float best_t = 0.0f;
    int best_k = -1;
    int cur = 0;
    int sp = 0;
    unsigned steps = 0;
    bool root_missed = false;
    int2 stack[kWideStack];  // (node ref, entry t bits): one 8-byte access per entry

    for (;;) {
        bool need = ray_idx == -1;
        unsigned need_mask = __ballot_sync(0xffffffffu, need);
        if (need_mask) {
            int leader = __ffs(need_mask) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(ray_counter, __popc(need_mask));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                unsigned idx = base + __popc(need_mask & lt);
                if (idx >= static_cast<unsigned>(nrays)) {
                    ray_idx = -2;
                } else {
                    ray_idx = static_cast<int>(idx);
                    ray = load_ray(rays, ray_idx);
                    sr = make_slab_ray(ray);
                    orr = make_octant_ray(sr);
                    best_t = ray.tmax;
                    best_k = -1;
                    sp = 0;
                    steps = 0;
                    float tn;
                    root_missed = bvh.n <= 0 || !slab_hit(sr, root, best_t, tn);
                    cur = bvh.n == 1 ? ~0 : 0;
                }
            }
        }
        if (__all_sync(0xffffffffu, ray_idx == -2)) break;

        bool done = false;
        if (ray_idx >= 0) {
            if (root_missed) done = true;
            for (int s = 0; s < budget && !done; ++s) {
                if (++steps > bound || cur >= bvh.n - 1 || ~cur >= bvh.n) {
                    atomicOr(error, kErrLoopBound);
                    best_k = -1;
                    best_t = ray.tmax;
                    done = true;
                    break;
                }
                bool pop = true;
                if (cur >= 0) {
                    const WideNode w = load_wide(bvh.wide, cur);
                    float t[4];
                    unsigned m = wide_test(w, sr, orr, best_t, t);
                    if (m) {
                        const int f = __ffs(m) - 1;
                        if (sp + __popc(m) - 1 > kWideStack) {
                            atomicOr(error, kErrStackOverflow);
                            best_k = -1;
                            best_t = ray.tmax;
                            done = true;
                            break;
                        }
#pragma unroll
                        for (int c = 3; c >= 1; --c) {
                            if (c > f && ((m >> c) & 1u)) {
                                stack[sp] = make_int2(wide_ref(w, c), __float_as_int(t[c]));
                                ++sp;
                            }
                        }
                        cur = wide_ref(w, f);
                        pop = false;
                    }
                } else if (float4 p0, p1, p2;
                           leaf_record_hit(bvh, ~cur, sr, orr, best_t, p0, p1, p2)) {
                    int k = ~cur;
                    float t, u, v;
                    if (moller_trumbore(ray.o, ray.d, make_f3(p0.x, p0.y, p0.z),
                                        make_f3(p1.x, p1.y, p1.z), make_f3(p2.x, p2.y, p2.z),
                                        t, u, v)
                        && t > ray.tmin && t < best_t) {
                        best_k = k;
                        best_t = t;
                        if (AnyHit) {
                            done = true;
                            break;
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
                    if (!resumed) done = true;
                }
            }
        }
        if (done) {
            int id = -1;
            if (best_k >= 0)
                id = __float_as_int(__ldg(reinterpret_cast<const float*>(bvh.tris + best_k) + 3));
            hit_id[ray_idx] = id;
            if (hit_t) hit_t[ray_idx] = best_k >= 0 ? best_t : INFINITY;
            ray_idx = -1;
        }
    }
}

// Totals of box and triangle tests over all rays (one atomic pair per warp).
__global__ void __launch_bounds__(kTraceThreads) k_trace_stats(BvhView bvh, const float4* rays,
                                                               int nrays,
                                                               unsigned long long* totals,
                                                               int* error) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    TraceCounts c;
    if (i < nrays) {
        ray3 ray = load_ray(rays, i);
        trace_one<false, true>(bvh, ray, error, &c);
    }
    unsigned long long b = c.boxes, t = c.tris;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        b += __shfl_xor_sync(0xffffffffu, b, off);
        t += __shfl_xor_sync(0xffffffffu, t, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(totals, b);
        atomicAdd(totals + 1, t);
    }
}

// ---------------------------------------------------------------- overlap

LUX_D bool boxes_overlap(const box3& a, const box3& b) {
    // AABB::overlaps (core/aabb.cuh:68-72).
    return !(b.lo.x > a.hi.x || b.hi.x < a.lo.x || b.lo.y > a.hi.y || b.hi.y < a.lo.y
             || b.lo.z > a.hi.z || b.hi.z < a.lo.z);
}

// Append one pair; the lanes that append in the same step share one atomic.
LUX_D void append_pair(int a, int b, int* pairs, long long max_pairs,
                       unsigned long long* counter) {
    unsigned active = __activemask();
    int lane = threadIdx.x & 31;
    int leader = __ffs(active) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(counter, static_cast<unsigned long long>(__popc(active)));
    base = __shfl_sync(active, base, leader);
    unsigned lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    unsigned long long slot = base + __popc(active & lt);
    if (slot < static_cast<unsigned long long>(max_pairs)) {
        reinterpret_cast<int2*>(pairs)[slot] = make_int2(a, b);
    }
}

// One thread per query leaf (sorted order of the query tree).  self: the query tree is
// the tree itself and only partners with a larger primitive id are reported.
template <bool Self>
__global__ void __launch_bounds__(kTraceThreads) k_overlap(BvhView tree, BvhView queries,
                                                           int* pairs, long long max_pairs,
                                                           unsigned long long* counter,
                                                           int* error) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= queries.n || tree.n <= 0) return;
    box3 qb = leaf_box(queries, q);
    int qid = queries.sorted_ids[q];
    if (!boxes_overlap(load_root(tree.root), qb)) return;
    int stack[kStack];
    int sp = 0;
    int cur = tree.n == 1 ? ~0 : 0;
    const long long bound = 2ll * tree.n + 64;
    for (long long step = 0;; ++step) {
        if (step > bound || cur >= tree.n - 1 || ~cur >= tree.n) {
            atomicOr(error, kErrLoopBound);
            return;
        }
        if (cur >= 0) {
            BvhNode nd = load_node(tree.nodes, cur);
            bool hl = boxes_overlap(node_left_box(nd), qb);
            bool hr = boxes_overlap(node_right_box(nd), qb);
            if (hl) {
                if (hr) {
                    if (sp < kStack) {
                        stack[sp++] = nd.ch.y;
                    } else {
                        atomicOr(error, kErrStackOverflow);
                        return;
                    }
                }
                cur = nd.ch.x;
                continue;
            }
            if (hr) {
                cur = nd.ch.y;
                continue;
            }
        } else {
            int pid = tree.sorted_ids[~cur];
            if (!Self || pid > qid) {
                if (Self) append_pair(qid, pid, pairs, max_pairs, counter);
                else append_pair(pid, qid, pairs, max_pairs, counter);
            }
        }
        if (sp == 0) break;
        cur = stack[--sp];
    }
}

template <bool AnyHit>
int launch_trace(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int nrays, int* hit_id,
                 float* hit_t) {
    if (nrays <= 0) return LUX_OK;
    const float4* r4 = reinterpret_cast<const float4*>(rays);
    if (ctx->trace_variant == kTraceWidePersistent || ctx->trace_variant == kTraceAuto) {
        if (int st = lbvh_ensure_wide(ctx, const_cast<lux_bvh*>(bvh))) return st;
        const int bps = occupancy_blocks(ctx, AnyHit ? kOccWideAny : kOccWideClosest,
                                         k_trace_wide_persistent<AnyHit>, kTraceThreads);
        int grid = std::min(ctx->sm_count * bps, (nrays + kTraceThreads - 1) / kTraceThreads);
        cudaError_t err = cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned), ctx->stream);
        if (err != cudaSuccess) return cuda_fail(err, "ray counter reset");
        k_trace_wide_persistent<AnyHit><<<grid, kTraceThreads, 0, ctx->stream>>>(
            bvh->view(), r4, nrays, hit_id, hit_t, ctx->d_counter, ctx->trace_budget,
            ctx->d_error);
        ctx->launches += 1;
        return cuda_fail(cudaGetLastError(), "k_trace_wide_persistent");
    }
    if (ctx->trace_variant == kTraceWide) {
        if (int st = lbvh_ensure_wide(ctx, const_cast<lux_bvh*>(bvh))) return st;
        int grid = (nrays + kTraceThreads - 1) / kTraceThreads;
        k_trace_wide<AnyHit><<<grid, kTraceThreads, 0, ctx->stream>>>(
            bvh->view(), r4, nrays, hit_id, hit_t, ctx->d_error);
        ctx->launches += 1;
        return cuda_fail(cudaGetLastError(), "k_trace_wide");
    }
    if (ctx->trace_variant == kTraceStatic) {
        int grid = (nrays + kTraceThreads - 1) / kTraceThreads;
        k_trace<AnyHit><<<grid, kTraceThreads, 0, ctx->stream>>>(bvh->view(), r4, nrays, hit_id,
                                                                 hit_t, ctx->d_error);
        ctx->launches += 1;
        return cuda_fail(cudaGetLastError(), "k_trace");
    }
    const int bps = occupancy_blocks(ctx, AnyHit ? kOccPersistAny : kOccPersistClosest,
                                     k_trace_persistent<AnyHit>, kTraceThreads);
    int grid = ctx->sm_count * bps;
    int needed = (nrays + kTraceThreads - 1) / kTraceThreads;
    if (grid > needed) grid = needed;
    cudaError_t err = cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned), ctx->stream);
    if (err != cudaSuccess) return cuda_fail(err, "ray counter reset");
    k_trace_persistent<AnyHit><<<grid, kTraceThreads, 0, ctx->stream>>>(
        bvh->view(), r4, nrays, hit_id, hit_t, ctx->d_counter, ctx->trace_budget, ctx->d_error);
    ctx->launches += 1;
    return cuda_fail(cudaGetLastError(), "k_trace_persistent");
}

}  // namespace

int trace_closest(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int nrays, int* hit_id,
                  float* hit_t) {
    return launch_trace<false>(ctx, bvh, rays, nrays, hit_id, hit_t);
}

int trace_any(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int nrays, int* hit_id) {
    return launch_trace<true>(ctx, bvh, rays, nrays, hit_id, nullptr);
}

int trace_stats(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int nrays,
                unsigned long long* totals) {
    if (nrays <= 0) return LUX_OK;
    int grid = (nrays + kTraceThreads - 1) / kTraceThreads;
    k_trace_stats<<<grid, kTraceThreads, 0, ctx->stream>>>(
        bvh->view(), reinterpret_cast<const float4*>(rays), nrays, totals, ctx->d_error);
    ctx->launches += 1;
    return cuda_fail(cudaGetLastError(), "k_trace_stats");
}

int overlap(lux_ctx* ctx, const lux_bvh* tree, const lux_bvh* queries, bool self, int* pairs,
            int64_t max_pairs, unsigned long long* d_found) {
    cudaError_t err = cudaMemsetAsync(d_found, 0, sizeof(unsigned long long), ctx->stream);
    if (err != cudaSuccess) return cuda_fail(err, "overlap counter");
    if (queries->n <= 0 || tree->n <= 0) return LUX_OK;
    int grid = (queries->n + kTraceThreads - 1) / kTraceThreads;
    if (self) {
        k_overlap<true><<<grid, kTraceThreads, 0, ctx->stream>>>(
            tree->view(), queries->view(), pairs, max_pairs, d_found, ctx->d_error);
    } else {
        k_overlap<false><<<grid, kTraceThreads, 0, ctx->stream>>>(
            tree->view(), queries->view(), pairs, max_pairs, d_found, ctx->d_error);
    }
    ctx->launches += 1;
    return cuda_fail(cudaGetLastError(), "k_overlap");
}

}  // namespace lux
