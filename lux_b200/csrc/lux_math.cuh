// Exact-rounding float helpers shared by the LBVH and path-tracing kernels.
//
// The reference's host build (x86-64, SSE2) evaluates every a*b+c as a rounded
// multiply followed by a rounded add; nvcc would contract such pairs into FMAs.  The
// parity-critical paths (Morton quantisation, slab test, Moller-Trumbore) therefore go
// through the _rn intrinsics below, which are never contracted, so device results are
// bit-identical to the host's.  Divisions and square roots use the default IEEE
// (correctly rounded) lowering.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define LUX_HD __host__ __device__ __forceinline__
#define LUX_D __device__ __forceinline__

namespace lux {

#ifdef __CUDA_ARCH__
LUX_HD float mul(float a, float b) { return __fmul_rn(a, b); }
LUX_HD float add(float a, float b) { return __fadd_rn(a, b); }
LUX_HD float sub(float a, float b) { return __fsub_rn(a, b); }
#else
LUX_HD float mul(float a, float b) { return a * b; }
LUX_HD float add(float a, float b) { return a + b; }
LUX_HD float sub(float a, float b) { return a - b; }
#endif

struct f3 {
    float x, y, z;
};

LUX_HD f3 make_f3(float x, float y, float z) { return f3{x, y, z}; }
LUX_HD f3 operator+(f3 a, f3 b) { return f3{add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)}; }
LUX_HD f3 operator-(f3 a, f3 b) { return f3{sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)}; }
LUX_HD f3 operator-(f3 a) { return f3{-a.x, -a.y, -a.z}; }
LUX_HD f3 operator*(f3 a, float s) { return f3{mul(a.x, s), mul(a.y, s), mul(a.z, s)}; }
LUX_HD f3 operator*(float s, f3 a) { return a * s; }
LUX_HD f3 operator*(f3 a, f3 b) { return f3{mul(a.x, b.x), mul(a.y, b.y), mul(a.z, b.z)}; }
// Left-to-right sum of products, as the reference's dot (core/vec3.cuh:44-46).
LUX_HD float dot(f3 a, f3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
// core/vec3.cuh:48-54.
LUX_HD f3 cross(f3 a, f3 b) {
    return f3{sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)),
              sub(mul(a.x, b.y), mul(a.y, b.x))};
}
LUX_HD float comp(f3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
LUX_HD f3 fmin3(f3 a, f3 b) { return f3{fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
LUX_HD f3 fmax3(f3 a, f3 b) { return f3{fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }

struct box3 {
    f3 lo, hi;
};

LUX_HD box3 box_union(box3 a, box3 b) { return box3{fmin3(a.lo, b.lo), fmax3(a.hi, b.hi)}; }

// triangle_bounds: expand the empty box by v0, v1, v2 (geometry/triangle.h:22-28).
LUX_HD box3 triangle_box(f3 v0, f3 v1, f3 v2) {
    box3 b;
    b.lo = fmin3(fmin3(make_f3(INFINITY, INFINITY, INFINITY), v0), fmin3(v1, v2));
    b.hi = fmax3(fmax3(make_f3(-INFINITY, -INFINITY, -INFINITY), v0), fmax3(v1, v2));
    // fminf/fmaxf are exact and order-free on non-NaN inputs, so the grouping above
    // equals the reference's sequential expand.
    return b;
}

// Ray in the form the traversal kernels use: inverse direction is NOT precomputed,
// because the reference computes 1/d inside the slab test (core/aabb.cuh:98) and the
// parallel-axis branch depends on d itself.
struct ray3 {
    f3 o;
    float tmin;
    f3 d;
    float tmax;
};

// Per-ray constants of the slab test: 1/d per axis (IEEE division) and the
// parallel-axis flags of core/aabb.cuh:92-96.  Hoisting them out of the node loop does
// not change any rounded value: the reference recomputes exactly these per node.
struct slab_ray {
    f3 o;
    f3 inv;
    unsigned parallel;  // bit a: |d_a| < 1e-12
    float tmin;
};

LUX_HD slab_ray make_slab_ray(const ray3& r) {
    slab_ray s;
    s.o = r.o;
    s.tmin = r.tmin;
    s.parallel = 0;
    float d[3] = {r.d.x, r.d.y, r.d.z};
    float inv[3];
    for (int a = 0; a < 3; ++a) {
        if (fabsf(d[a]) < 1e-12f) {
            s.parallel |= 1u << a;
            inv[a] = 0.0f;
        } else {
            inv[a] = 1.0f / d[a];
        }
    }
    s.inv = make_f3(inv[0], inv[1], inv[2]);
    return s;
}

// Slab test of core/aabb.cuh:84-109 split into its t_max-free part: returns the entry
// distance tn = max(t_min, per-axis entries) and the exit tf = min(per-axis exits).
// The box is hit under a current t_max iff (!rejected && tn <= min(t_max, tf)), which
// is the reference's final `t_near > t_far` decision (t_near only grows and t_far only
// shrinks across axes, so its early exits change nothing).
LUX_HD bool slab_entry(const slab_ray& r, const box3& b, float& tn, float& tf) {
    tn = r.tmin;
    tf = INFINITY;
    float lo[3] = {b.lo.x, b.lo.y, b.lo.z};
    float hi[3] = {b.hi.x, b.hi.y, b.hi.z};
    float o[3] = {r.o.x, r.o.y, r.o.z};
    float inv[3] = {r.inv.x, r.inv.y, r.inv.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (r.parallel & (1u << a)) {
            if (o[a] < lo[a] || o[a] > hi[a]) return false;
            continue;
        }
        float t0 = mul(sub(lo[a], o[a]), inv[a]);
        float t1 = mul(sub(hi[a], o[a]), inv[a]);
        if (inv[a] < 0.0f) {
            float t = t0;
            t0 = t1;
            t1 = t;
        }
        tn = fmaxf(tn, t0);
        tf = fminf(tf, t1);
    }
    return true;
}

LUX_HD bool slab_hit(const slab_ray& r, const box3& b, float tmax, float& tn) {
    float tf;
    if (!slab_entry(r, b, tn, tf)) return false;
    return !(tn > fminf(tmax, tf));
}

// Octant form of the same slab test for rays with no parallel axis: the near plane of
// axis a is lo_a when 1/d_a > 0 and hi_a otherwise, which yields exactly the values the
// reference's per-box swap (core/aabb.cuh:100-104) produces, without the compare and
// swap per box.  neg bit a: 1/d_a < 0.
struct octant_ray {
    f3 o;
    f3 inv;
    float tmin;
    unsigned neg;
};

LUX_HD octant_ray make_octant_ray(const slab_ray& s) {
    octant_ray r;
    r.o = s.o;
    r.inv = s.inv;
    r.tmin = s.tmin;
    r.neg = (s.inv.x < 0.0f ? 1u : 0u) | (s.inv.y < 0.0f ? 2u : 0u) | (s.inv.z < 0.0f ? 4u : 0u);
    return r;
}

LUX_HD bool octant_hit(const octant_ray& r, const box3& b, float tmax, float& tn) {
    float nx = (r.neg & 1u) ? b.hi.x : b.lo.x, fx = (r.neg & 1u) ? b.lo.x : b.hi.x;
    float ny = (r.neg & 2u) ? b.hi.y : b.lo.y, fy = (r.neg & 2u) ? b.lo.y : b.hi.y;
    float nz = (r.neg & 4u) ? b.hi.z : b.lo.z, fz = (r.neg & 4u) ? b.lo.z : b.hi.z;
    float t0x = mul(sub(nx, r.o.x), r.inv.x), t1x = mul(sub(fx, r.o.x), r.inv.x);
    float t0y = mul(sub(ny, r.o.y), r.inv.y), t1y = mul(sub(fy, r.o.y), r.inv.y);
    float t0z = mul(sub(nz, r.o.z), r.inv.z), t1z = mul(sub(fz, r.o.z), r.inv.z);
    tn = fmaxf(fmaxf(r.tmin, t0x), fmaxf(t0y, t0z));
    float tf = fminf(fminf(tmax, t1x), fminf(t1y, t1z));
    return !(tn > tf);
}

// Moller-Trumbore (geometry/triangle.h:33-52) on the triangle's vertices: the edges
// e1 = v1 - v0 and e2 = v2 - v0 are the same rounded differences the reference forms.
// Returns the raw t; the caller applies t_min < t < t_max.
LUX_HD bool moller_trumbore(const f3& o, const f3& d, f3 v0, f3 v1, f3 v2, float& t,
                            float& u, float& v) {
    const f3 e1 = v1 - v0;
    const f3 e2 = v2 - v0;
    f3 h = cross(d, e2);
    float a = dot(e1, h);
    if (fabsf(a) < 1e-7f) return false;
    float f = 1.0f / a;
    f3 s = o - v0;
    u = mul(f, dot(s, h));
    if (u < 0.0f || u > 1.0f) return false;
    f3 q = cross(s, e1);
    v = mul(f, dot(d, q));
    if (v < 0.0f || add(u, v) > 1.0f) return false;
    t = mul(f, dot(e2, q));
    return true;
}

// ------------------------------------------------------------------ Morton codes

// Spread the low 10 bits so that bit k lands on bit 3k (bvh/gpu_bvh.cu:46-53).
LUX_HD uint32_t spread10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0xff0000ffu;
    v = (v | (v << 8)) & 0x0f00f00fu;
    v = (v | (v << 4)) & 0xc30c30c3u;
    v = (v | (v << 2)) & 0x49249249u;
    return v;
}

// 21-bit version for 63-bit codes (no reference counterpart; same construction).
LUX_HD uint64_t spread21(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// Box centroid (core/aabb.cuh:20).
LUX_HD f3 box_centroid(const box3& b) { return (b.lo + b.hi) * 0.5f; }

// Normalised offset of centroid c inside the scene box (core/aabb.cuh:74-81).
LUX_HD f3 centroid_offset_of(f3 c, const box3& root) {
    f3 d = root.hi - root.lo;
    return make_f3(d.x > 0 ? (c.x - root.lo.x) / d.x : 0.5f,
                   d.y > 0 ? (c.y - root.lo.y) / d.y : 0.5f,
                   d.z > 0 ? (c.z - root.lo.z) / d.z : 0.5f);
}

// Normalised centroid offset inside the scene box (core/aabb.cuh:20, 74-81).
LUX_HD f3 centroid_offset(const box3& b, const box3& root) {
    return centroid_offset_of(box_centroid(b), root);
}

// quantize_morton_coord (bvh/gpu_bvh.cu:61-64) with a general scale.
LUX_HD uint32_t quantize(float v, float scale, float maxv) {
    v = fmaxf(0.0f, fminf(maxv, mul(v, scale)));
    return static_cast<uint32_t>(v);
}

LUX_HD uint32_t morton30_of(f3 centroid, const box3& root) {
    f3 off = centroid_offset_of(centroid, root);
    return (spread10(quantize(off.x, 1024.0f, 1023.0f)) << 2)
         | (spread10(quantize(off.y, 1024.0f, 1023.0f)) << 1)
         | spread10(quantize(off.z, 1024.0f, 1023.0f));
}

LUX_HD uint64_t morton63_of(f3 centroid, const box3& root) {
    f3 off = centroid_offset_of(centroid, root);
    return (spread21(quantize(off.x, 2097152.0f, 2097151.0f)) << 2)
         | (spread21(quantize(off.y, 2097152.0f, 2097151.0f)) << 1)
         | spread21(quantize(off.z, 2097152.0f, 2097151.0f));
}

LUX_HD uint32_t morton30(const box3& b, const box3& root) { return morton30_of(box_centroid(b), root); }
LUX_HD uint64_t morton63(const box3& b, const box3& root) { return morton63_of(box_centroid(b), root); }

// Order-preserving float <-> uint32 map for atomicMin/atomicMax reductions.
LUX_HD uint32_t float_to_ordered(float f) {
#ifdef __CUDA_ARCH__
    uint32_t u = __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
#endif
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

LUX_HD float ordered_to_float(uint32_t o) {
    uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

}  // namespace lux

// Validation builds only: with LUX_ROUNDED_DOUBLE_MATH (lux_b200/build.py compiles the
// sources that way into lux_b200/liblux_gpu_dmath.so, beside the product library) the
// float sinf, cosf, powf, acosf and atan2f calls are evaluated in double precision and
// rounded to float, on the device and on the host alike.  A reference build with the same
// substitution (oracle/rounded_double_math.h) then rounds those calls identically, which
// isolates the last-bit differences between CUDA's and glibc's float functions as the
// cause of the path tracer's few per-sample mismatches.  The product library never
// defines it.
#ifdef LUX_ROUNDED_DOUBLE_MATH
__host__ __device__ inline float lux_rd_sinf(float x) { return static_cast<float>(sin(static_cast<double>(x))); }
__host__ __device__ inline float lux_rd_cosf(float x) { return static_cast<float>(cos(static_cast<double>(x))); }
__host__ __device__ inline float lux_rd_powf(float x, float y) {
    return static_cast<float>(pow(static_cast<double>(x), static_cast<double>(y)));
}
__host__ __device__ inline float lux_rd_acosf(float x) { return static_cast<float>(acos(static_cast<double>(x))); }
__host__ __device__ inline float lux_rd_atan2f(float y, float x) {
    return static_cast<float>(atan2(static_cast<double>(y), static_cast<double>(x)));
}
#define sinf lux_rd_sinf
#define cosf lux_rd_cosf
#define powf lux_rd_powf
#define acosf lux_rd_acosf
#define atan2f lux_rd_atan2f
#endif
