// Test infrastructure only: force-included (g++ -include) into the validation build of
// the reference harness (oracle/_ref/libluxref_dmath.so, oracle/build.py) so that the
// reference's float sinf, cosf, powf, acosf and atan2f calls are evaluated in double
// precision and rounded to float, exactly as lux_b200/liblux_gpu_dmath.so evaluates them
// on the device (LUX_ROUNDED_DOUBLE_MATH in lux_b200/csrc/lux_math.cuh).  tanf (the
// camera's field of view, computed on the host on both sides with glibc) is left alone.
// The standard headers are included first so that only the reference's own calls are
// renamed.
#pragma once

#include <math.h>

#include <cmath>
#include <complex>
#include <random>

static inline float lux_rd_sinf(float x) { return static_cast<float>(sin(static_cast<double>(x))); }
static inline float lux_rd_cosf(float x) { return static_cast<float>(cos(static_cast<double>(x))); }
static inline float lux_rd_powf(float x, float y) {
    return static_cast<float>(pow(static_cast<double>(x), static_cast<double>(y)));
}
static inline float lux_rd_acosf(float x) { return static_cast<float>(acos(static_cast<double>(x))); }
static inline float lux_rd_atan2f(float y, float x) {
    return static_cast<float>(atan2(static_cast<double>(y), static_cast<double>(x)));
}
#define sinf lux_rd_sinf
#define cosf lux_rd_cosf
#define powf lux_rd_powf
#define acosf lux_rd_acosf
#define atan2f lux_rd_atan2f
