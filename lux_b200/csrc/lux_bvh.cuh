// Device-side LBVH layout shared by the build, refit, traversal and overlap kernels.
//
// Internal node i is Karras node i (the same numbering as bvh/gpu_bvh.cu:151-180 and
// the host tree of bvh/cpu_lbvh_builder.h).  Unlike the reference's 32-byte
// one-box-per-node stackless records (bvh/bvh_device.cuh:12-17), a node here carries
// the boxes of BOTH children, so a traversal step tests two boxes per 64-byte fetch
// and never fetches a leaf node at all.
#pragma once

#include "lux_math.cuh"

namespace lux {

// Child handle: >= 0 internal node index; < 0 leaf, sorted leaf index k = ~handle.
LUX_HD bool is_leaf_handle(int h) { return h < 0; }

struct alignas(16) BvhNode {
    float4 a;  // left.lo.x  left.lo.y  left.lo.z  left.hi.x
    float4 b;  // left.hi.y  left.hi.z  right.lo.x right.lo.y
    float4 c;  // right.lo.z right.hi.x right.hi.y right.hi.z
    int4 ch;   // left handle, right handle, unused, unused
};
static_assert(sizeof(BvhNode) == 64, "one node is one 64-byte record");

// Triangle in Morton order: its three vertices, primitive id in p0.w.  The walks form
// the edges v1 - v0 and v2 - v0 when they test it (the reference's Moller-Trumbore
// rounds the same two differences), and a triangle BVH's leaf box is the triangle's box
// (triangle_box of these vertices), so a leaf's exact box comes from the record itself.
struct alignas(16) TriRecord {
    float4 p0;  // v0.xyz, primitive id (int bits)
    float4 p1;  // v1.xyz, 0
    float4 p2;  // v2.xyz, 0
};

LUX_HD box3 node_left_box(const BvhNode& n) {
    return box3{make_f3(n.a.x, n.a.y, n.a.z), make_f3(n.a.w, n.b.x, n.b.y)};
}
LUX_HD box3 node_right_box(const BvhNode& n) {
    return box3{make_f3(n.b.z, n.b.w, n.c.x), make_f3(n.c.y, n.c.z, n.c.w)};
}

// 4-wide node of binary internal node i: its grandchildren in left-first order, a leaf
// child standing for itself, so 2 to 4 children.  One is built for every internal node;
// a walk from the root enters only those at even binary depth.  Child boxes are stored
// quantised to 8 bits per plane on a per-axis power-of-two grid s = 2^e whose points are
// integer multiples of s (the grid starts at k * s, the node's lower corner rounded down
// to the grid), rounded outward, so each decoded box contains the exact one; the node is
// 64 bytes.  Plane q decodes to (k + q) * s, which is a float exactly (|k| <= 2^22), as
// one fused multiply-add fma(2^23 + q, s, c) with c = (k - 2^23) * s: the 2^23 + q is the
// plane byte placed in the mantissa of 2^23 by one byte permute.  Decoded boxes only
// steer the walk: a leaf is accepted by the exact test of its own box when the walk
// reaches it.
//   q0 = c.xyz, meta (bits 0-23: biased exponents x, y, z; 24-26: child count;
//        27: unbounded, every child passes)
//   q1 = lo.x, lo.y, lo.z, hi.x bytes of children 0..3 (byte c of each word: child c)
//   q2 = hi.y, hi.z bytes, child handles 0, 1
//   q3 = child handles 2, 3, 0, 0
struct alignas(16) WideNode {
    float4 q0, q1, q2, q3;
};
static_assert(sizeof(WideNode) == 64, "one wide node is one 64-byte record");

constexpr unsigned kWideUnbounded = 1u << 27;

LUX_D float wide_scale(unsigned biased) { return __int_as_float(static_cast<int>(biased) << 23); }

// Plane byte q as the float 2^23 + q (exact for q < 2^23).
LUX_D float wide_biased(unsigned q) { return __uint_as_float(0x4B000000u | q); }

// Decoded plane (k + q) * 2^e of grid offset c = (k - 2^23) * 2^e: the fused
// multiply-add's exact result is a float, so it is returned unrounded.
LUX_D float wide_decode(float c, unsigned q, float scale) {
    return __fmaf_rn(wide_biased(q), scale, c);
}

// Non-owning view passed by value into kernels.
struct BvhView {
    const BvhNode* nodes = nullptr;     // n - 1 internal nodes
    const WideNode* wide = nullptr;     // n - 1 wide nodes (ray queries), indexed as nodes
    const TriRecord* tris = nullptr;    // n triangles in sorted order (triangle BVHs)
    const int* sorted_ids = nullptr;    // n: input index of sorted leaf k
    const int* leaf_parent = nullptr;   // n: (parent << 1) | slot, -1 for a lone leaf
    const float* root = nullptr;        // 6 floats: union of all boxes
    int n = 0;
    // Leaf boxes are the triangles' own boxes (BVHs built from triangles); false for box
    // BVHs with attached triangles, whose leaf boxes are the caller's boxes.
    bool leaf_is_triangle_box = false;
};

LUX_D box3 load_root(const float* root) {
    return box3{make_f3(root[0], root[1], root[2]), make_f3(root[3], root[4], root[5])};
}

LUX_D BvhNode load_node(const BvhNode* nodes, int i) {
    BvhNode n;
    const float4* p = reinterpret_cast<const float4*>(nodes + i);
    n.a = __ldg(p + 0);
    n.b = __ldg(p + 1);
    n.c = __ldg(p + 2);
    n.ch = __ldg(reinterpret_cast<const int4*>(p + 3));
    return n;
}

// Box of sorted leaf k: the slot its parent stores (for a one-primitive tree, the root).
// Only the slot's 24 bytes are read.
LUX_D box3 leaf_box(const BvhView& v, int k) {
    int code = v.leaf_parent[k];
    if (code < 0 || (code >> 1) >= v.n - 1) return load_root(v.root);
    const float* f = reinterpret_cast<const float*>(v.nodes + (code >> 1));
    if (code & 1) {
        const float2 a = __ldg(reinterpret_cast<const float2*>(f + 6));
        const float4 b = __ldg(reinterpret_cast<const float4*>(f + 8));
        return box3{make_f3(a.x, a.y, b.x), make_f3(b.y, b.z, b.w)};
    }
    const float4 a = __ldg(reinterpret_cast<const float4*>(f));
    const float2 b = __ldg(reinterpret_cast<const float2*>(f + 4));
    return box3{make_f3(a.x, a.y, a.z), make_f3(a.w, b.x, b.y)};
}

// Device error word bits (ctx-owned, read back by the host at synchronisation points).
enum : int {
    kErrClimbBound = 1,      // bottom-up pass exceeded its level bound
    kErrStackOverflow = 2,   // traversal stack overflow
    kErrLoopBound = 4,       // a bounded loop ran out of iterations
    kErrQueueOverflow = 8,   // a work queue exceeded capacity
};

}  // namespace lux
