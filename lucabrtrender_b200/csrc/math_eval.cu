// Diagnostic: the rasteriser's own exp (with and without its range checks),
// log, sRGB, cut-off and float-to-half functions evaluated on the device, so tests can compare their bits with the host's.
#include "../../include/lrt_raster.h"
#include "kernels.cuh"
#include "raster_common.cuh"

namespace lrt {
namespace {

__global__ void math_eval_kernel(int fn, const float* __restrict__ x, float* __restrict__ y, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = x[i];
    float out;
    switch (fn) {
        case 0: out = lrt_exp(v); break;
        case 1: out = lrt_log(v); break;
        case 2: out = srgb_to_linear(v); break;
        case 3: out = cutoff_power(v); break;
        case 4: out = __uint_as_float(float_to_half(v)); break;
        case 5: out = __uint_as_float(pack_halves(v, -0.5f * v)); break;
        case 6: out = lrt_exp_in_range(v); break;   // for -87 <= v <= 88 only
        default: out = NAN; break;
    }
    y[i] = out;
}

}  // namespace

cudaError_t launch_math_eval(int fn, const float* x, float* y, uint32_t n, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    math_eval_kernel<<<(n + 255) / 256, 256, 0, stream>>>(fn, x, y, n);
    return cudaGetLastError();
}

}  // namespace lrt

extern "C" int lrt_math_eval(int fn, const void* x, void* y, uint32_t n, void* stream) {
    if (fn < 0 || fn > 6 || (n > 0 && (x == nullptr || y == nullptr))) return LRT_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = lrt::launch_math_eval(fn, static_cast<const float*>(x), static_cast<float*>(y), n, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? LRT_OK : LRT_DEVICE_FAILURE;
}
