// The photometric L1 loss of a training step, one kernel each way (no
// reference counterpart: the reference renders only). colour is the
// rasteriser's float4 image (linear, premultiplied), target a float3 image
// of the same pixels; the loss is mean |colour.rgb - target| over pixels and
// channels, summed in a fixed order (per block, then over the blocks), so it
// does not change from run to run. Its gradient with respect to colour is
// sign(colour.rgb - target) / (3 pixels), scaled by the loss's own incoming
// gradient (read on the device, so the backward needs no host sync); alpha
// gets zero.
#include "kernels.cuh"
#include "raster_common.cuh"

namespace lrt {
namespace {

constexpr uint32_t kLossThreads = 256;
constexpr uint32_t kLossBlocks = 148 * 4;

template <bool kChained>
__global__ void __launch_bounds__(kLossThreads)
l1_partial_kernel(const float4* __restrict__ colour, const float* __restrict__ target, uint32_t pixels,
                  float* __restrict__ partials) {
    chained_entry<kChained>();
    __shared__ float sWarp[kLossThreads / 32];
    float s = 0.0f;
    for (uint32_t i = blockIdx.x * kLossThreads + threadIdx.x; i < pixels; i += gridDim.x * kLossThreads) {
        const float4 c = __ldg(colour + i);
        const float tr = __ldg(target + 3 * static_cast<size_t>(i)), tg = __ldg(target + 3 * static_cast<size_t>(i) + 1),
                    tb = __ldg(target + 3 * static_cast<size_t>(i) + 2);
        s += fabsf(c.x - tr) + fabsf(c.y - tg) + fabsf(c.z - tb);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31u) == 0) sWarp[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = 0.0f;
        for (uint32_t w = 0; w < kLossThreads / 32; ++w) b += sWarp[w];
        partials[blockIdx.x] = b;
    }
}

template <bool kChained>
__global__ void l1_total_kernel(const float* __restrict__ partials, uint32_t count, float scale,
                                float* __restrict__ loss) {
    chained_entry<kChained>();
    __shared__ float sWarp[32];
    float s = 0.0f;
    for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) s += partials[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31u) == 0) sWarp[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) t += sWarp[w];
        *loss = t * scale;
    }
}

template <bool kChained>
__global__ void __launch_bounds__(kLossThreads)
l1_grad_kernel(const float4* __restrict__ colour, const float* __restrict__ target, uint32_t pixels, float scale,
               const float* __restrict__ gradLoss, float4* __restrict__ gradColour) {
    chained_entry<kChained>();
    const float g = scale * (gradLoss != nullptr ? __ldg(gradLoss) : 1.0f);
    for (uint32_t i = blockIdx.x * kLossThreads + threadIdx.x; i < pixels; i += gridDim.x * kLossThreads) {
        const float4 c = __ldg(colour + i);
        const float d0 = c.x - __ldg(target + 3 * static_cast<size_t>(i));
        const float d1 = c.y - __ldg(target + 3 * static_cast<size_t>(i) + 1);
        const float d2 = c.z - __ldg(target + 3 * static_cast<size_t>(i) + 2);
        auto sgn = [](float d) { return d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f); };
        gradColour[i] = make_float4(sgn(d0) * g, sgn(d1) * g, sgn(d2) * g, 0.0f);
    }
}

}  // namespace

size_t l1_scratch_bytes() { return kLossBlocks * sizeof(float); }

cudaError_t launch_l1_loss(const float4* colour, const float* target, uint32_t pixels, float* scratch, float* loss,
                           cudaStream_t stream) {
    const float scale = pixels > 0 ? 1.0f / (3.0f * static_cast<float>(pixels)) : 0.0f;
    const ChainScope chain(pixels >= kChainMinPixels);
    cudaError_t e = launch_chained(l1_partial_kernel<true>, l1_partial_kernel<false>, dim3(kLossBlocks), dim3(kLossThreads), 0, stream, colour, target,
                                   pixels, scratch);
    if (e != cudaSuccess) return e;
    return launch_chained(l1_total_kernel<true>, l1_total_kernel<false>, dim3(1), dim3(256), 0, stream, static_cast<const float*>(scratch),
                          kLossBlocks, scale, loss);
}

cudaError_t launch_l1_grad(const float4* colour, const float* target, uint32_t pixels, const float* gradLoss,
                           float4* gradColour, cudaStream_t stream) {
    if (pixels == 0) return cudaSuccess;
    const float scale = 1.0f / (3.0f * static_cast<float>(pixels));
    const ChainScope chain(pixels >= kChainMinPixels);
    return launch_chained(l1_grad_kernel<true>, l1_grad_kernel<false>, dim3(kLossBlocks), dim3(kLossThreads), 0, stream, colour, target, pixels,
                          scale, gradLoss, gradColour);
}

}  // namespace lrt
