// Drop-in shims: the reference's own C++ interfaces for the GPU LBVH
// (bvh/gpu_bvh.cuh:50-61, bvh/bvh_overlap.cuh:21-23) and for the wavefront integrator
// (integrator/wavefront_pt.cuh:14-28, integrator/integrator.h:15-22), implemented over
// the C ABI of liblux_gpu.so (include/lux_gpu.h).  A maintainer compiles
// gpu_bvh_lux.cpp and wavefront_pt_lux.cu into the reference in place of
// bvh/gpu_bvh.cu, bvh/bvh_overlap.cu and integrator/wavefront_*.cu, against the
// reference's own headers, and links liblux_gpu.so.
//
// Threading and devices follow the reference's GPU code: one host thread, device 0.  The
// shims share one library context, created on first use and kept for the life of the
// process.  Errors become std::runtime_error, as the reference's CUDA checks throw
// (core/cuda_check.cuh:7-27).
#pragma once

#include <stdexcept>
#include <string>

#include "lux_gpu.h"

namespace lux_shim {

// The process's library context (device 0, its own stream).
lux_ctx* context();

inline void check(int status, const char* what) {
    if (status != LUX_OK) throw std::runtime_error(std::string(what) + ": " + lux_last_error());
}

}  // namespace lux_shim
