// Test and measurement infrastructure only: the reference's OWN GPU LBVH code behind a
// small C ABI, compiled by oracle/build.py with nvcc for sm_100a from the reference
// sources where they lie (bvh/gpu_bvh.cu is included below so its file-local kernels can
// be timed alone; bvh/bvh_overlap.cu is a second translation unit) into
// oracle/_ref/libluxrefgpu.so.  The flags are the reference's stock CUDA configuration
// (C++20, -O3, LUX_ENABLE_CUDA=1, nvcc's default contraction).  Tests compare its hits
// with lux_b200's; bench.py times it as the reference's GPU code on the same B200 and
// workload.  Nothing in the product loads this library.
//
// Reference entry points exercised (paths relative to the reference's src/):
//   build_gpu_lbvh                 bvh/gpu_bvh.cu:535-595
//   refit_gpu_lbvh                 bvh/gpu_bvh.cu:597-613
//   intersect_gpu_bvh_stackless    bvh/gpu_bvh.cu:893-915 (host vectors in and out)
//   trace_rays_kernel              bvh/gpu_bvh.cu:371-384 (the same kernel, inputs resident)
//   query_aabb_overlaps_cross      bvh/bvh_overlap.cu

#include "bvh/gpu_bvh.cu"

#include <chrono>
#include <cstring>
#include <exception>

#include "bvh/bvh_overlap.cuh"

namespace {

std::string g_refgpu_error;

std::vector<BvhBuildPrimitive> box_primitives(const float* prims, int n, bool triangles) {
    std::vector<BvhBuildPrimitive> out;
    out.reserve(n);
    for (int i = 0; i < n; ++i) {
        AABB bounds;
        if (triangles) {
            const float* t = prims + size_t(i) * 9;
            Triangle tri{vec3(t[0], t[1], t[2]), vec3(t[3], t[4], t[5]), vec3(t[6], t[7], t[8])};
            bounds = triangle_bounds(tri);
        } else {
            const float* b = prims + size_t(i) * 6;
            bounds = AABB(vec3(b[0], b[1], b[2]), vec3(b[3], b[4], b[5]));
        }
        out.push_back(BvhBuildPrimitive{bounds, bounds.centroid(), i, -1, -1, i,
                                        PrimitiveKind::Triangle});
    }
    return out;
}

std::vector<Triangle> triangle_list(const float* tris, int n) {
    std::vector<Triangle> out(n);
    for (int i = 0; i < n; ++i) {
        const float* t = tris + size_t(i) * 9;
        out[i] = Triangle{vec3(t[0], t[1], t[2]), vec3(t[3], t[4], t[5]), vec3(t[6], t[7], t[8])};
    }
    return out;
}

// Ray record of include/lux_gpu.h: origin.xyz, t_min, direction.xyz, t_max.
std::vector<Ray> ray_list(const float* rays, int n) {
    std::vector<Ray> out;
    out.reserve(n);
    for (int i = 0; i < n; ++i) {
        const float* r = rays + size_t(i) * 8;
        out.push_back(Ray(vec3(r[0], r[1], r[2]), vec3(r[4], r[5], r[6]), r[3], r[7]));
    }
    return out;
}

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

double median(std::vector<double> v) {
    std::sort(v.begin(), v.end());
    return v.empty() ? 0.0 : v[v.size() / 2];
}

}  // namespace

extern "C" {

const char* refgpu_last_error(void) { return g_refgpu_error.c_str(); }

// Closest hits of nrays rays against ntri triangles through the reference's public GPU
// API (build_gpu_lbvh, then intersect_gpu_bvh_stackless).  Returns 0, or -1 with
// refgpu_last_error set when the reference threw.
int refgpu_trace(const float* tris, int ntri, const float* rays, int nrays, int32_t* hit_id,
                 float* hit_t) {
    try {
        GpuBvh bvh = build_gpu_lbvh(box_primitives(tris, ntri, true));
        std::vector<GpuRayHit> hits =
            intersect_gpu_bvh_stackless(bvh, triangle_list(tris, ntri), ray_list(rays, nrays));
        for (int i = 0; i < nrays; ++i) {
            hit_id[i] = hits[i].primitive_id;
            hit_t[i] = hits[i].t;
        }
        return 0;
    } catch (const std::exception& e) {
        g_refgpu_error = e.what();
        return -1;
    }
}

// The LBVH microbench step on the reference's GPU code, each phase timed `reps` times
// after one untimed run (medians, ms; host clock around each call, which synchronises):
//   times[0] build_gpu_lbvh over the triangles (host primitive vector in)
//   times[1] intersect_gpu_bvh_stackless (host triangles and rays in, hits out)
//   times[2] trace_rays_kernel alone on device-resident inputs (CUDA events, L2
//            flushed before each launch by a 256 MiB write)
//   times[3] refit_gpu_lbvh with the jittered triangles
//   times[4] build_gpu_lbvh over the query boxes
//   times[5] query_aabb_overlaps_cross(triangle tree, query tree, max_pairs)
// found receives the overlap count of the last run.  The host-side preparation of the
// reference's input vectors (primitive records, Triangle and Ray lists) is not timed.
int refgpu_microbench(const float* tris, int ntri, const float* rays, int nrays,
                      const float* refit_tris, const float* queries, int nqueries,
                      int max_pairs, int reps, double* times, int64_t* found) {
    try {
        const std::vector<BvhBuildPrimitive> prims = box_primitives(tris, ntri, true);
        const std::vector<BvhBuildPrimitive> refit_prims = box_primitives(refit_tris, ntri, true);
        const std::vector<BvhBuildPrimitive> query_prims = box_primitives(queries, nqueries, false);
        const std::vector<Triangle> tri_list = triangle_list(tris, ntri);
        const std::vector<Ray> ray_vec = ray_list(rays, nrays);
        std::vector<double> t[6];
        thrust::device_vector<Triangle> d_tris = tri_list;
        thrust::device_vector<Ray> d_rays = ray_vec;
        thrust::device_vector<GpuRayHit> d_hits(ray_vec.size());
        thrust::device_vector<unsigned char> flush(size_t(256) << 20);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        for (int rep = 0; rep <= reps; ++rep) {
            double a = now_ms();
            GpuBvh bvh = build_gpu_lbvh(prims);
            synchronize_cuda_or_throw("build");
            double b = now_ms();
            std::vector<GpuRayHit> hits = intersect_gpu_bvh_stackless(bvh, tri_list, ray_vec);
            double c = now_ms();
            LUX_CUDA_CHECK(cudaMemset(thrust::raw_pointer_cast(flush.data()), rep & 0xff,
                                      flush.size()));
            cudaEventRecord(e0);
            trace_rays_kernel<<<grid_size(nrays), kBlockSize>>>(
                bvh.device_view(), thrust::raw_pointer_cast(d_tris.data()),
                thrust::raw_pointer_cast(d_rays.data()), thrust::raw_pointer_cast(d_hits.data()),
                nrays);
            cudaEventRecord(e1);
            synchronize_cuda_or_throw("trace_rays_kernel");
            float kernel_ms = 0;
            cudaEventElapsedTime(&kernel_ms, e0, e1);
            double d = now_ms();
            if (!refit_gpu_lbvh(bvh, refit_prims)) throw std::runtime_error("refit refused");
            synchronize_cuda_or_throw("refit");
            double e = now_ms();
            GpuBvh qbvh = build_gpu_lbvh(query_prims);
            synchronize_cuda_or_throw("query build");
            double f = now_ms();
            OverlapQueryResult overlap = query_aabb_overlaps_cross(bvh, qbvh, max_pairs);
            double g = now_ms();
            *found = overlap.found_count;
            if (rep == 0) continue;
            t[0].push_back(b - a);
            t[1].push_back(c - b);
            t[2].push_back(kernel_ms);
            t[3].push_back(e - d);
            t[4].push_back(f - e);
            t[5].push_back(g - f);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        for (int k = 0; k < 6; ++k) times[k] = median(t[k]);
        return 0;
    } catch (const std::exception& e) {
        g_refgpu_error = e.what();
        return -1;
    }
}

}  // extern "C"
