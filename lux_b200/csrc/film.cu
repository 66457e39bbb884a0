// Film encoding on the device: the pixel transforms of the reference's image writers
// (film/ppm.h:37-79, film/pfm.h:27-40) applied to a film of per-pixel sums.
//   LUX_FILM_PPM8         sum / spp, Reinhard c / (1 + c), clamp to [0, 1],
//                         255.999 * c^(1/2.2) truncated to a byte; rows top first
//   LUX_FILM_PPM8_LINEAR  sum / spp clamped to [0, 1], 255.999 * c truncated
//   LUX_FILM_PFM          sum / spp as float32, rows bottom first (the PFM order)
// 1 / spp is formed once (film_inv_sample_count, film/film.h:11-13) and multiplied in,
// as the writers do.  The gamma uses CUDA's powf, which may round a last bit
// differently from the host's, so a byte can differ by one where the exact value sits
// on a quantisation boundary.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/lux_gpu.h"
#include "lux_internal.h"

namespace lux {
namespace {

constexpr int kEncodeThreads = 256;

__device__ float clamp01f(float v) { return fmaxf(0.0f, fminf(1.0f, v)); }

__global__ void __launch_bounds__(kEncodeThreads) k_encode(const float* film, int width,
                                                           int height, float inv_spp, int format,
                                                           void* out) {
    const long long n = static_cast<long long>(width) * height;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        float c[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) c[a] = __fmul_rn(film[3 * i + a], inv_spp);
        if (format == LUX_FILM_PFM) {
            const long long y = i / width, x = i - y * width;
            float* o = static_cast<float*>(out) + 3 * ((height - 1 - y) * width + x);
#pragma unroll
            for (int a = 0; a < 3; ++a) o[a] = c[a];
            continue;
        }
        unsigned char* o = static_cast<unsigned char*>(out) + 3 * i;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float v = c[a];
            if (format == LUX_FILM_PPM8) {
                v = clamp01f(__fdiv_rn(v, __fadd_rn(1.0f, v)));
                v = __fmul_rn(255.999f, powf(v, 1.0f / 2.2f));
            } else {
                v = __fmul_rn(255.999f, clamp01f(v));
            }
            o[a] = static_cast<unsigned char>(v);
        }
    }
}

}  // namespace
}  // namespace lux

extern "C" int lux_film_encode(lux_ctx* ctx, const float* film_sum, int32_t width,
                               int32_t height, int32_t spp, int32_t format, void* out) {
    if (!ctx || !film_sum || !out) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    if (width <= 0 || height <= 0) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "empty film");
    if (format != LUX_FILM_PPM8 && format != LUX_FILM_PPM8_LINEAR && format != LUX_FILM_PFM)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "unknown film format");
    if (cudaError_t err = cudaSetDevice(ctx->device)) return lux::cuda_fail(err, "cudaSetDevice");
    const size_t pixels = static_cast<size_t>(width) * height;
    const size_t in_bytes = pixels * 3 * sizeof(float);
    const size_t out_bytes = pixels * 3 * (format == LUX_FILM_PFM ? sizeof(float) : 1);
    auto on_device = [](const void* p) {
        cudaPointerAttributes a{};
        bool dev = cudaPointerGetAttributes(&a, p) == cudaSuccess &&
                   (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged);
        cudaGetLastError();
        return dev;
    };
    const bool in_dev = on_device(film_sum), out_dev = on_device(out);
    void* d_in = const_cast<float*>(film_sum);  // replaced by staging when on the host
    void* d_out = out;
    cudaStream_t s = ctx->stream;
    cudaError_t err = cudaSuccess;
    if (!in_dev) err = cudaMallocAsync(&d_in, in_bytes, s);
    if (err == cudaSuccess && !out_dev) err = cudaMallocAsync(&d_out, out_bytes, s);
    if (err == cudaSuccess && !in_dev)
        err = cudaMemcpyAsync(d_in, film_sum, in_bytes, cudaMemcpyHostToDevice, s);
    if (err != cudaSuccess) {
        if (!in_dev && d_in != film_sum) cudaFreeAsync(d_in, s);
        if (!out_dev && d_out != out) cudaFreeAsync(d_out, s);
        return lux::cuda_fail(err, "film staging");
    }
    const float inv_spp = spp > 0 ? 1.0f / static_cast<float>(spp) : 0.0f;
    const int grid = static_cast<int>(
        std::min<size_t>((pixels + lux::kEncodeThreads - 1) / lux::kEncodeThreads,
                         static_cast<size_t>(ctx->sm_count) * 8));
    lux::k_encode<<<grid, lux::kEncodeThreads, 0, s>>>(static_cast<const float*>(d_in), width,
                                                      height, inv_spp, format, d_out);
    ctx->launches += 1;
    err = cudaGetLastError();
    if (err == cudaSuccess && !out_dev)
        err = cudaMemcpyAsync(out, d_out, out_bytes, cudaMemcpyDeviceToHost, s);
    if (!in_dev) cudaFreeAsync(d_in, s);
    if (!out_dev) cudaFreeAsync(d_out, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    return lux::cuda_fail(err, "film encode");
}
