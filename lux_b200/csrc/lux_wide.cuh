// Ray walk over the 4-wide nodes (WideNode), shared by the LBVH ray queries and the path
// tracer's TLAS and BLAS searches.
//
// Results are those of the reference's stackless walk (intersect_bvh_device_impl,
// bvh/bvh_device.cuh:43-90): leaves in left-first order, a box accepted when its slab
// entry does not exceed min(exit, best t), a triangle when t_min < t < best t.  The walk
// descends through the decoded (outward-rounded) child boxes, entering the first child
// that passes and deferring the others with their entry distances, resumed while the
// entry does not exceed the best t.  Decoded boxes contain the exact ones and the slab
// bounds are monotone in the box, so every leaf the reference reaches is reached here, in
// the same order; each leaf is then accepted by the exact test of its own box under the
// best t of that moment, which is the reference's verdict (its ancestors' exact boxes
// pass whenever the leaf's does).  The leaves tested and the best hit after each are
// therefore the reference's, so hit ids and t agree bit for bit.
#pragma once

#include "lux_bvh.cuh"

namespace lux {

constexpr int kWideStack = 112;  // three deferred children per wide level

LUX_D WideNode load_wide(const WideNode* wide, int i) {
    const float4* p = reinterpret_cast<const float4*>(wide + i);
    WideNode w;
    w.q0 = __ldg(p);
    w.q1 = __ldg(p + 1);
    w.q2 = __ldg(p + 2);
    w.q3 = __ldg(p + 3);
    return w;
}

LUX_D int wide_ref(const WideNode& w, int c) {
    return __float_as_int(c == 0 ? w.q2.z : c == 1 ? w.q2.w : c == 2 ? w.q3.x : w.q3.y);
}

// Slab verdict of one box under t_max (octant form when no axis is parallel).
LUX_D bool child_hit(const box3& b, const slab_ray& sr, const octant_ray& orr, float tmax,
                     float& tn) {
    return sr.parallel == 0 ? octant_hit(orr, b, tmax, tn) : slab_hit(sr, b, tmax, tn);
}

// Byte c of a packed plane word as the float 2^23 + byte (wide_biased): one byte permute
// into the mantissa of 2^23, full-rate ALU work where an integer-to-float conversion would
// use the slower conversion pipe (24 of them per node visit).
LUX_D float biased_byte(unsigned word, int c) {
    return __uint_as_float(__byte_perm(word, 0x4B000000u, 0x7540u + c));
}

// Hit mask of the node's decoded child boxes (bit c: child c) under t_max and each
// child's entry t.  Decoded boxes contain the exact ones, so a child whose exact box
// passes always passes here.
LUX_D unsigned wide_test(const WideNode& w, const slab_ray& sr, const octant_ray& orr,
                         float tmax, float tn[4]) {
    const unsigned meta = __float_as_uint(w.q0.w);
    const unsigned count = (meta >> 24) & 7u;
    const unsigned live = (1u << count) - 1u;
    if (meta & kWideUnbounded) {
#pragma unroll
        for (int c = 0; c < 4; ++c) tn[c] = sr.tmin;
        return live;
    }
    const float sx = wide_scale(meta & 255u);
    const float sy = wide_scale((meta >> 8) & 255u);
    const float sz = wide_scale((meta >> 16) & 255u);
    const unsigned lx = __float_as_uint(w.q1.x), ly = __float_as_uint(w.q1.y);
    const unsigned lz = __float_as_uint(w.q1.z), hx = __float_as_uint(w.q1.w);
    const unsigned hy = __float_as_uint(w.q2.x), hz = __float_as_uint(w.q2.y);
    unsigned mask = 0;
    if (sr.parallel == 0) {
        // octant_hit on each decoded box, with its near / far choice made once per axis
        // on the packed words (the same bytes, so the same decoded planes and t values).
        const unsigned nxq = (orr.neg & 1u) ? hx : lx, fxq = (orr.neg & 1u) ? lx : hx;
        const unsigned nyq = (orr.neg & 2u) ? hy : ly, fyq = (orr.neg & 2u) ? ly : hy;
        const unsigned nzq = (orr.neg & 4u) ? hz : lz, fzq = (orr.neg & 4u) ? lz : hz;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            // Decoded planes (wide_decode), each one fused multiply-add.
            const float nx = __fmaf_rn(biased_byte(nxq, c), sx, w.q0.x);
            const float fx = __fmaf_rn(biased_byte(fxq, c), sx, w.q0.x);
            const float ny = __fmaf_rn(biased_byte(nyq, c), sy, w.q0.y);
            const float fy = __fmaf_rn(biased_byte(fyq, c), sy, w.q0.y);
            const float nz = __fmaf_rn(biased_byte(nzq, c), sz, w.q0.z);
            const float fz = __fmaf_rn(biased_byte(fzq, c), sz, w.q0.z);
            const float t0x = mul(sub(nx, orr.o.x), orr.inv.x), t1x = mul(sub(fx, orr.o.x), orr.inv.x);
            const float t0y = mul(sub(ny, orr.o.y), orr.inv.y), t1y = mul(sub(fy, orr.o.y), orr.inv.y);
            const float t0z = mul(sub(nz, orr.o.z), orr.inv.z), t1z = mul(sub(fz, orr.o.z), orr.inv.z);
            tn[c] = fmaxf(fmaxf(orr.tmin, t0x), fmaxf(t0y, t0z));
            const float tf = fminf(fminf(tmax, t1x), fminf(t1y, t1z));
            if (!(tn[c] > tf)) mask |= 1u << c;
        }
        return mask & live;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int sh = 8 * c;
        box3 b{make_f3(wide_decode(w.q0.x, (lx >> sh) & 255u, sx),
                       wide_decode(w.q0.y, (ly >> sh) & 255u, sy),
                       wide_decode(w.q0.z, (lz >> sh) & 255u, sz)),
               make_f3(wide_decode(w.q0.x, (hx >> sh) & 255u, sx),
                       wide_decode(w.q0.y, (hy >> sh) & 255u, sy),
                       wide_decode(w.q0.z, (hz >> sh) & 255u, sz))};
        if (child_hit(b, sr, orr, tmax, tn[c])) mask |= 1u << c;
    }
    return mask & live;
}

// The reference's verdict on sorted leaf k's own box under the current best t.
LUX_D bool leaf_hit(const BvhView& b, int k, const slab_ray& sr, const octant_ray& orr,
                    float best_t) {
    float tn;
    return child_hit(leaf_box(b, k), sr, orr, best_t, tn);
}

// Sorted leaf k's triangle record (p0, p1, p2) and the verdict on the leaf's exact box.
// In a BVH built from triangles the leaf box is the triangle's own box, formed here from
// the record's vertices exactly as the build formed it, so the leaf costs one 48-byte
// record load and no parent-slot load.
LUX_D bool leaf_record_hit(const BvhView& b, int k, const slab_ray& sr, const octant_ray& orr,
                           float best_t, float4& p0, float4& p1, float4& p2) {
    const float4* tp = reinterpret_cast<const float4*>(b.tris + k);
    p0 = __ldg(tp);
    p1 = __ldg(tp + 1);
    p2 = __ldg(tp + 2);
    if (!b.leaf_is_triangle_box) return leaf_hit(b, k, sr, orr, best_t);
    float tn;
    return child_hit(triangle_box(make_f3(p0.x, p0.y, p0.z), make_f3(p1.x, p1.y, p1.z),
                                  make_f3(p2.x, p2.y, p2.z)),
                     sr, orr, best_t, tn);
}

// Walks bvh from its root for a ray with slab constants sr; leaf(k, p0, p1, p2, best_t)
// tests sorted leaf k (its triangle record p0..p2), may lower best_t, and returns true to
// end the walk (any-hit).  Returns false after setting an error bit (loop bound or stack
// overflow).
template <typename Leaf>
LUX_D bool wide_walk(const BvhView& b, const slab_ray& sr, float& best_t, int* error,
                     Leaf&& leaf) {
    if (b.n <= 0) return true;
    float tn0;
    if (!slab_hit(sr, load_root(b.root), best_t, tn0)) return true;
    const octant_ray orr = make_octant_ray(sr);
    int2 stack[kWideStack];  // (node ref, entry t bits)
    int sp = 0;
    int cur = b.n == 1 ? ~0 : 0;
    const long long bound = 2ll * b.n + 64;
    for (long long step = 0;; ++step) {
        if (step > bound || cur >= b.n - 1 || ~cur >= b.n) {
            atomicOr(error, kErrLoopBound);
            return false;
        }
        bool descend = false;
        if (cur >= 0) {
            const WideNode w = load_wide(b.wide, cur);
            float t[4];
            unsigned m = wide_test(w, sr, orr, best_t, t);
            if (m) {
                const int f = __ffs(m) - 1;
                if (sp + __popc(m) - 1 > kWideStack) {
                    atomicOr(error, kErrStackOverflow);
                    return false;
                }
#pragma unroll
                for (int c = 3; c >= 1; --c) {
                    if (c > f && ((m >> c) & 1u)) {
                        stack[sp] = make_int2(wide_ref(w, c), __float_as_int(t[c]));
                        ++sp;
                    }
                }
                cur = wide_ref(w, f);
                descend = true;
            }
        } else {
            float4 p0, p1, p2;
            if (leaf_record_hit(b, ~cur, sr, orr, best_t, p0, p1, p2) &&
                leaf(~cur, p0, p1, p2, best_t))
                return true;
        }
        if (!descend) {
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
    return true;
}

}  // namespace lux
