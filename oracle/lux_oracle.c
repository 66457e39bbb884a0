/*
 * ORACLE -- test infrastructure only.
 *
 * A plain-C CPU restatement of the reference's LBVH algorithms, used by tests/ as the
 * checker for the CUDA path and by bench.py's cpu_baseline leg.  The product never
 * links, loads or calls this code.  Parity of this restatement is pinned against the
 * reference's own host code (oracle/_ref/libluxref.so, built from the reference
 * sources by oracle/build.py) and against the committed fixtures in tests/golden/.
 *
 * File:line citations are relative to the reference's src/ directory.
 *
 * Arithmetic is IEEE single precision without contraction (compiled with
 * -ffp-contract=off), matching the reference host build on x86-64.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_LEAF 0x80000000u
#define ORC_INDEX 0x7fffffffu

typedef struct { float x, y, z; } v3;

static inline v3 v3_make(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 v3_sub(v3 a, v3 b) { return v3_make(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline float v3_dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 v3_cross(v3 a, v3 b) {
    return v3_make(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float comp(v3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

/* ---------------------------------------------------------------- bounds */

/* triangle_bounds: geometry/triangle.h:22-28 (expand from the empty box with fminf/fmaxf). */
void orc_triangle_bounds(const float* tris, int n, float* bounds) {
    for (int i = 0; i < n; ++i) {
        const float* t = tris + (size_t)i * 9;
        float* b = bounds + (size_t)i * 6;
        for (int a = 0; a < 3; ++a) {
            float lo = INFINITY, hi = -INFINITY;
            for (int k = 0; k < 3; ++k) {
                lo = fminf(lo, t[k * 3 + a]);
                hi = fmaxf(hi, t[k * 3 + a]);
            }
            b[a] = lo;
            b[3 + a] = hi;
        }
    }
}

/* Union of all primitive boxes: bvh/cpu_lbvh_builder.h:202-205. */
void orc_root_bounds(const float* bounds, int n, float* root) {
    for (int a = 0; a < 3; ++a) { root[a] = INFINITY; root[3 + a] = -INFINITY; }
    for (int i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            root[a] = fminf(root[a], bounds[(size_t)i * 6 + a]);
            root[3 + a] = fmaxf(root[3 + a], bounds[(size_t)i * 6 + 3 + a]);
        }
    }
}

/* ---------------------------------------------------------------- Morton codes */

/* Spread the low 10 bits of v so that bit k lands on bit 3k
 * (bvh/cpu_lbvh_builder.h:37-44). */
static uint32_t spread10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0xff0000ffu;
    v = (v | (v << 8)) & 0x0f00f00fu;
    v = (v | (v << 4)) & 0xc30c30c3u;
    v = (v | (v << 2)) & 0x49249249u;
    return v;
}

/* Spread the low 21 bits of v so that bit k lands on bit 3k (63-bit codes; the
 * reference has no 63-bit path, this is the same construction at 21 bits/axis). */
static uint64_t spread21(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

/* Centroid and normalised offset: core/aabb.cuh:20 and 74-81. */
static void centroid_offset(const float* b, const float* root, float* off) {
    for (int a = 0; a < 3; ++a) {
        float c = (b[a] + b[3 + a]) * 0.5f;
        float d = root[3 + a] - root[a];
        off[a] = d > 0 ? (c - root[a]) / d : 0.5f;
    }
}

/* quantize_morton_coord: bvh/cpu_lbvh_builder.h:50-53, generalised to `scale`. */
static uint32_t quantize(float v, float scale, float maxv) {
    v = fmaxf(0.0f, fminf(maxv, v * scale));
    return (uint32_t)v;
}

/* centroid_to_morton: bvh/cpu_lbvh_builder.h:55-61 (x << 2 | y << 1 | z). */
void orc_morton30(const float* bounds, int n, const float* root, uint32_t* codes) {
    for (int i = 0; i < n; ++i) {
        float off[3];
        centroid_offset(bounds + (size_t)i * 6, root, off);
        codes[i] = (spread10(quantize(off[0], 1024.0f, 1023.0f)) << 2)
                 | (spread10(quantize(off[1], 1024.0f, 1023.0f)) << 1)
                 | spread10(quantize(off[2], 1024.0f, 1023.0f));
    }
}

void orc_morton63(const float* bounds, int n, const float* root, uint64_t* codes) {
    for (int i = 0; i < n; ++i) {
        float off[3];
        centroid_offset(bounds + (size_t)i * 6, root, off);
        codes[i] = (spread21(quantize(off[0], 2097152.0f, 2097151.0f)) << 2)
                 | (spread21(quantize(off[1], 2097152.0f, 2097151.0f)) << 1)
                 | spread21(quantize(off[2], 2097152.0f, 2097151.0f));
    }
}

/* ---------------------------------------------------------------- stable sort */

/* Stable ordering by code, ties in input order: std::stable_sort in
 * bvh/cpu_lbvh_builder.h:212-216.  Bottom-up merge sort on indices. */
void orc_stable_order(const uint64_t* codes, int n, int32_t* order) {
    int32_t* tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) order[i] = i;
    for (int width = 1; width < n; width *= 2) {
        for (int lo = 0; lo < n; lo += 2 * width) {
            int mid = lo + width < n ? lo + width : n;
            int hi = lo + 2 * width < n ? lo + 2 * width : n;
            int i = lo, j = mid, k = lo;
            while (i < mid && j < hi) {
                if (codes[order[j]] < codes[order[i]]) tmp[k++] = order[j++];
                else tmp[k++] = order[i++];
            }
            while (i < mid) tmp[k++] = order[i++];
            while (j < hi) tmp[k++] = order[j++];
        }
        memcpy(order, tmp, sizeof(int32_t) * (size_t)n);
    }
    free(tmp);
}

/* ---------------------------------------------------------------- Karras 2012 */

typedef struct {
    const uint64_t* codes; /* sorted */
    int n;
    int wide; /* 0: 30-bit codes keyed with the index (merged 64-bit key); 1: 63-bit */
} prefix_ctx;

static int clz64(uint64_t v) { return v ? __builtin_clzll(v) : 64; }
static int clz32(uint32_t v) { return v ? __builtin_clz(v) : 32; }

/* common_prefix: bvh/cpu_lbvh_builder.h:82-86 (merged key (code << 32) | index).  For
 * 63-bit codes the key no longer fits 64 bits, so the index bits extend the prefix
 * only when the codes are equal. */
static int delta(const prefix_ctx* c, int i, int j) {
    if (!c->wide) {
        uint64_t ki = (c->codes[i] << 32) | (uint32_t)i;
        uint64_t kj = (c->codes[j] << 32) | (uint32_t)j;
        return clz64(ki ^ kj);
    }
    uint64_t x = c->codes[i] ^ c->codes[j];
    if (x) return clz64(x);
    return 64 + clz32((uint32_t)i ^ (uint32_t)j);
}

/* determine_range: bvh/cpu_lbvh_builder.h:88-117. */
static void determine_range(const prefix_ctx* c, int idx, int* first, int* last) {
    int n = c->n;
    if (idx == 0) { *first = 0; *last = n - 1; return; }
    int dl = delta(c, idx, idx - 1);
    int dr = delta(c, idx, idx + 1);
    int dir = dr > dl ? 1 : -1;
    int dmin = dl < dr ? dl : dr;
    int lmax = 2;
    for (;;) {
        int cand = idx + dir * lmax;
        if (cand < 0 || cand >= n) break;
        if (delta(c, idx, cand) <= dmin) break;
        lmax <<= 1;
    }
    int len = 0;
    for (int step = lmax >> 1; step > 0; step >>= 1) {
        int cand = idx + (len + step) * dir;
        if (cand < 0 || cand >= n) continue;
        if (delta(c, idx, cand) > dmin) len += step;
    }
    int other = idx + len * dir;
    if (dir < 0) { *first = other; *last = idx; } else { *first = idx; *last = other; }
}

/* find_split: bvh/cpu_lbvh_builder.h:119-133. */
static int find_split(const prefix_ctx* c, int first, int last) {
    int node_delta = delta(c, first, last);
    int split = first;
    int stride = last - first;
    do {
        stride = (stride + 1) >> 1;
        int mid = split + stride;
        if (mid < last && delta(c, first, mid) > node_delta) split = mid;
    } while (stride > 1);
    return split;
}

/*
 * Full host LBVH: bvh/cpu_lbvh_builder.h:163-259.
 *
 * Inputs: primitive boxes (n x 6 floats) and the Morton width (30 or 63).
 * Outputs (any may be NULL):
 *   sorted_codes[n]      codes in sorted order (u64 even for 30-bit)
 *   sorted_ids[n]        input index of each sorted leaf
 *   child[2*(n-1)]       Karras children, bit 31 = leaf, low bits = index
 *   node_left/right[2n-1] the reference CpuBvhTree layout: internal nodes 0..n-2, leaf
 *                        k at n-1+k; -1 on leaves
 *   node_bounds[(2n-1)*6]
 * Returns the node count (2n-1), 0 for n == 0.
 */
int orc_lbvh_build(const float* bounds, int n, int morton_bits, uint64_t* sorted_codes,
                   int32_t* sorted_ids, uint32_t* child, int32_t* node_left,
                   int32_t* node_right, float* node_bounds) {
    if (n <= 0) return 0;
    int count = 2 * n - 1;
    if (n == 1) {
        if (sorted_codes) sorted_codes[0] = 0;
        if (sorted_ids) sorted_ids[0] = 0;
        if (node_left) node_left[0] = -1;
        if (node_right) node_right[0] = -1;
        if (node_bounds) memcpy(node_bounds, bounds, sizeof(float) * 6);
        return 1;
    }
    float root[6];
    orc_root_bounds(bounds, n, root);
    uint64_t* codes = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    if (morton_bits == 63) {
        orc_morton63(bounds, n, root, codes);
    } else {
        uint32_t* c32 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
        orc_morton30(bounds, n, root, c32);
        for (int i = 0; i < n; ++i) codes[i] = c32[i];
        free(c32);
    }
    int32_t* order = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    orc_stable_order(codes, n, order);
    uint64_t* sc = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    for (int i = 0; i < n; ++i) sc[i] = codes[order[i]];
    if (sorted_codes) memcpy(sorted_codes, sc, sizeof(uint64_t) * (size_t)n);
    if (sorted_ids) memcpy(sorted_ids, order, sizeof(int32_t) * (size_t)n);

    prefix_ctx ctx = {sc, n, morton_bits == 63};
    uint32_t* ch = (uint32_t*)malloc(sizeof(uint32_t) * 2 * (size_t)(n - 1));
    for (int i = 0; i < n - 1; ++i) {
        int first, last;
        determine_range(&ctx, i, &first, &last);
        int split = find_split(&ctx, first, last);
        ch[2 * i] = (first == split ? ORC_LEAF : 0u) | (uint32_t)split;
        ch[2 * i + 1] = (last == split + 1 ? ORC_LEAF : 0u) | (uint32_t)(split + 1);
    }
    if (child) memcpy(child, ch, sizeof(uint32_t) * 2 * (size_t)(n - 1));

    int ni = n - 1;
    if (node_left || node_right) {
        for (int i = 0; i < ni; ++i) {
            for (int s = 0; s < 2; ++s) {
                uint32_t c = ch[2 * i + s];
                int idx = (c & ORC_LEAF) ? ni + (int)(c & ORC_INDEX) : (int)c;
                if (s == 0 && node_left) node_left[i] = idx;
                if (s == 1 && node_right) node_right[i] = idx;
            }
        }
        for (int k = 0; k < n; ++k) {
            if (node_left) node_left[ni + k] = -1;
            if (node_right) node_right[ni + k] = -1;
        }
    }
    if (node_bounds) {
        /* fill_internal_bounds: bvh/cpu_lbvh_builder.h:139-159, iterative post-order. */
        for (int k = 0; k < n; ++k)
            memcpy(node_bounds + (size_t)(ni + k) * 6, bounds + (size_t)order[k] * 6,
                   sizeof(float) * 6);
        int* stack = (int*)malloc(sizeof(int) * 2 * (size_t)n);
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            int top = stack[sp - 1];
            int node = top & 0x3fffffff;
            int done = top & 0x40000000;
            if (!done) {
                stack[sp - 1] = node | 0x40000000;
                for (int s = 1; s >= 0; --s) {
                    uint32_t c = ch[2 * node + s];
                    if (!(c & ORC_LEAF)) stack[sp++] = (int)c;
                }
                continue;
            }
            --sp;
            float* out = node_bounds + (size_t)node * 6;
            const float* lb;
            const float* rb;
            uint32_t l = ch[2 * node], r = ch[2 * node + 1];
            lb = node_bounds + (size_t)((l & ORC_LEAF) ? ni + (int)(l & ORC_INDEX) : (int)l) * 6;
            rb = node_bounds + (size_t)((r & ORC_LEAF) ? ni + (int)(r & ORC_INDEX) : (int)r) * 6;
            for (int a = 0; a < 3; ++a) {
                out[a] = fminf(lb[a], rb[a]);
                out[3 + a] = fmaxf(lb[3 + a], rb[3 + a]);
            }
        }
        free(stack);
    }
    free(ch);
    free(sc);
    free(order);
    free(codes);
    return count;
}

/* ---------------------------------------------------------------- traversal */

typedef struct {
    v3 o, d;
    float tmin, tmax;
} ray_t;

/* AABB::intersect slab test: core/aabb.cuh:84-109. */
static int slab(const float* b, const ray_t* r) {
    float t_near = r->tmin, t_far = r->tmax;
    for (int i = 0; i < 3; ++i) {
        float d = comp(r->d, i), o = comp(r->o, i);
        if (fabsf(d) < 1e-12f) {
            if (o < b[i] || o > b[3 + i]) return 0;
            continue;
        }
        float inv = 1.0f / d;
        float a = (b[i] - o) * inv;
        float c = (b[3 + i] - o) * inv;
        if (inv < 0) { float t = a; a = c; c = t; }
        t_near = fmaxf(t_near, a);
        t_far = fminf(t_far, c);
        if (t_near > t_far) return 0;
    }
    return 1;
}

/* AABB::overlaps: core/aabb.cuh:68-72. */
static int overlaps(const float* a, const float* b) {
    return !(b[0] > a[3] || b[3] < a[0] || b[1] > a[4] || b[4] < a[1] || b[2] > a[5]
             || b[5] < a[2]);
}

/* Moller-Trumbore: geometry/triangle.h:33-52. */
static int tri_hit(const float* t, const ray_t* r, float* tout) {
    v3 v0 = v3_make(t[0], t[1], t[2]);
    v3 e1 = v3_sub(v3_make(t[3], t[4], t[5]), v0);
    v3 e2 = v3_sub(v3_make(t[6], t[7], t[8]), v0);
    v3 h = v3_cross(r->d, e2);
    float a = v3_dot(e1, h);
    if (fabsf(a) < 1e-7f) return 0;
    float f = 1.0f / a;
    v3 s = v3_sub(r->o, v0);
    float u = f * v3_dot(s, h);
    if (u < 0.0f || u > 1.0f) return 0;
    v3 q = v3_cross(s, e1);
    float v = f * v3_dot(r->d, q);
    if (v < 0.0f || u + v > 1.0f) return 0;
    float tt = f * v3_dot(e2, q);
    *tout = tt;
    return tt > r->tmin && tt < r->tmax;
}

/*
 * Closest hit in the reference GPU order: the stackless preorder walk of
 * bvh/bvh_device.cuh:43-90 (left child first, strict t < best, t_max shrinks on each
 * hit), expressed over the Karras children.  A preorder walk with escape links visits
 * exactly the nodes a left-first depth-first walk visits, so this is written as one.
 *
 * Node boxes: node_bounds in the CpuBvhTree layout from orc_lbvh_build.  any_hit != 0
 * stops at the first hit (occlusion query).  ignored: primitive id skipped (-1 none).
 * stats (optional, 2 x int64 per ray): box tests, triangle tests.
 */
void orc_trace(const float* tris, const float* node_bounds, const uint32_t* child,
               const int32_t* sorted_ids, int n, const float* rays, int nrays, int any_hit,
               int ignored, int32_t* hit_id, float* hit_t, int64_t* stats) {
    int ni = n - 1;
    int* stack = (int*)malloc(sizeof(int) * 128);
    for (int q = 0; q < nrays; ++q) {
        const float* rr = rays + (size_t)q * 8;
        /* record: origin.xyz, t_min, direction.xyz, t_max */
        ray_t r = {v3_make(rr[0], rr[1], rr[2]), v3_make(rr[4], rr[5], rr[6]), rr[3], rr[7]};
        int best = -1;
        float best_t = r.tmax;
        int64_t boxes = 0, tests = 0;
        if (n > 0) {
            int sp = 0;
            /* Node handle: >= 0 internal index, < 0 leaf -(k+1). */
            stack[sp++] = n == 1 ? -1 : 0;
            while (sp > 0) {
                int h = stack[--sp];
                int leaf = h < 0;
                int k = leaf ? -h - 1 : h;
                const float* b = node_bounds + (size_t)(leaf ? ni + k : k) * 6;
                ++boxes;
                if (!slab(b, &r)) continue;
                if (leaf) {
                    int pid = sorted_ids[k];
                    if (pid == ignored) continue;
                    ++tests;
                    float t;
                    if (tri_hit(tris + (size_t)pid * 9, &r, &t) && t < best_t) {
                        best = pid;
                        best_t = t;
                        r.tmax = t;
                        if (any_hit) break;
                    }
                    continue;
                }
                uint32_t l = child[2 * k], rc = child[2 * k + 1];
                stack[sp++] = (rc & ORC_LEAF) ? -(int)(rc & ORC_INDEX) - 1 : (int)rc;
                stack[sp++] = (l & ORC_LEAF) ? -(int)(l & ORC_INDEX) - 1 : (int)l;
            }
        }
        hit_id[q] = best;
        hit_t[q] = best >= 0 ? best_t : INFINITY;
        if (stats) { stats[2 * q] = boxes; stats[2 * q + 1] = tests; }
    }
    free(stack);
}

/*
 * Overlap pairs.  Self (bvh/bvh_overlap.cu:25-105): for every primitive a, every leaf
 * primitive b whose box overlaps a's box with b > a (ids are input indices here).
 * Cross (bvh/bvh_overlap.cu:107-184): every (left b, right a) with overlapping boxes.
 * Written as the brute-force check of bvh/bvh_validation.h:195-236 would be, but
 * through the tree so that it stays fast at 10^6 boxes; pair sets are order free.
 * Returns the total pair count; writes at most max_pairs pairs (a, b) as int32 x 2.
 */
int64_t orc_overlap(const float* tree_node_bounds, const uint32_t* child,
                    const int32_t* sorted_ids, int n, const float* query_bounds, int nq,
                    int self, int32_t* pairs, int64_t max_pairs) {
    int ni = n - 1;
    int64_t found = 0;
    int* stack = (int*)malloc(sizeof(int) * 128);
    for (int q = 0; q < nq && n > 0; ++q) {
        const float* qb = query_bounds + (size_t)q * 6;
        int sp = 0;
        stack[sp++] = n == 1 ? -1 : 0;
        while (sp > 0) {
            int h = stack[--sp];
            int leaf = h < 0;
            int k = leaf ? -h - 1 : h;
            if (!overlaps(tree_node_bounds + (size_t)(leaf ? ni + k : k) * 6, qb)) continue;
            if (leaf) {
                int pid = sorted_ids[k];
                if (self && pid <= q) continue;
                if (found < max_pairs) {
                    pairs[2 * found] = self ? q : pid;
                    pairs[2 * found + 1] = self ? pid : q;
                }
                ++found;
                continue;
            }
            uint32_t l = child[2 * k], rc = child[2 * k + 1];
            stack[sp++] = (rc & ORC_LEAF) ? -(int)(rc & ORC_INDEX) - 1 : (int)rc;
            stack[sp++] = (l & ORC_LEAF) ? -(int)(l & ORC_INDEX) - 1 : (int)l;
        }
    }
    free(stack);
    return found;
}
