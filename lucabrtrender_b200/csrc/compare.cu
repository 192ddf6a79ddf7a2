// Parity metrics on the device (modules/render/src/ReferenceRenderer.cpp:
// 248-396): two renders compared without reading either back.
//
// compareImages (shaders/lrt/reference/image_compare.slang:20-51): per
// pixel, the largest difference of 8-bit sRGB code values over r, g, b
// (premultiplied) and of the 8-bit alpha, into a 256-bin histogram. The
// reference counts per row and then reduces the rows; here every pixel is one
// thread, each block keeps its own histogram in shared memory and adds it to
// the frame's with one atomic per non-empty bin. Counts are integers, so the
// result does not depend on the order.
//
// compareHdr (image_compare_hdr.slang:20-60): per pixel the largest relative
// channel difference, binned eight to an octave from 2^-16, and the relative
// squared error. The error is summed exactly as the reference does: each row
// in pixel order with compensated (Kahan) addition, then the rows in order.
//
// countDifferent (image_compare_hdr.slang:62-80): how many of two uint
// buffers' entries differ.
#include "kernels.cuh"
#include "raster_common.cuh"

namespace lrt {
namespace {

constexpr uint32_t kCompareThreads = 256;

__device__ __forceinline__ float saturate(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// image_compare.slang:20-25
__device__ __forceinline__ int code_of(float linear) {
    const float c = saturate(linear);
    const float e = c <= 0.0031308f ? c * 12.92f : 1.055f * lrt_pow(c, 1.0f / 2.4f) - 0.055f;
    return static_cast<int>(roundf(e * 255.0f));
}

__global__ void __launch_bounds__(kCompareThreads)
compare_images_kernel(const float4* __restrict__ a, const float4* __restrict__ b, uint32_t pixels,
                      uint32_t* __restrict__ histogram) {
    __shared__ uint32_t sHist[256];
    sHist[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * kCompareThreads + threadIdx.x; i < pixels; i += gridDim.x * kCompareThreads) {
        const float4 pa = __ldg(a + i), pb = __ldg(b + i);
        int worst = abs(code_of(pa.x) - code_of(pb.x));
        worst = max(worst, abs(code_of(pa.y) - code_of(pb.y)));
        worst = max(worst, abs(code_of(pa.z) - code_of(pb.z)));
        worst = max(worst, abs(static_cast<int>(roundf(saturate(pa.w) * 255.0f)) -
                               static_cast<int>(roundf(saturate(pb.w) * 255.0f))));
        atomicAdd(&sHist[worst], 1u);
    }
    __syncthreads();
    if (sHist[threadIdx.x] != 0) atomicAdd(&histogram[threadIdx.x], sHist[threadIdx.x]);
}

// log2 by the library's own log (the bins must agree with the CPU side bit for bit).
__device__ __forceinline__ float log2_of(float x) { return lrt_log(x) / 0.693147182464599609375f; }

__global__ void __launch_bounds__(kCompareThreads)
hdr_histogram_kernel(const float4* __restrict__ a, const float4* __restrict__ b, uint32_t pixels,
                     uint32_t* __restrict__ histogram) {
    __shared__ uint32_t sHist[256];
    sHist[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * kCompareThreads + threadIdx.x; i < pixels; i += gridDim.x * kCompareThreads) {
        const float4 pa = __ldg(a + i), pb = __ldg(b + i);
        const float va[4] = {pa.x, pa.y, pa.z, pa.w}, vb[4] = {pb.x, pb.y, pb.z, pb.w};
        float worst = 0.0f;
#pragma unroll
        for (int c = 0; c < 4; ++c) worst = fmaxf(worst, fabsf(va[c] - vb[c]) / fmaxf(fabsf(vb[c]), 1e-3f));
        const uint32_t bin = worst <= 0.0f
                                 ? 0u
                                 : static_cast<uint32_t>(fminf(fmaxf(floorf((log2_of(worst) + 16.0f) * 8.0f) + 1.0f,
                                                                     1.0f), 255.0f));
        atomicAdd(&sHist[bin], 1u);
    }
    __syncthreads();
    if (sHist[threadIdx.x] != 0) atomicAdd(&histogram[threadIdx.x], sHist[threadIdx.x]);
}

// Compensated addition as image_compare_hdr.slang:48-51 writes it.
__device__ __forceinline__ void kahan_add(float& sum, float& carry, float term) {
    const float t = sum + term;
    carry += fabsf(sum) >= fabsf(term) ? (sum - t) + term : (term - t) + sum;
    sum = t;
}

__global__ void hdr_rows_kernel(const float4* __restrict__ a, const float4* __restrict__ b, uint32_t width,
                                uint32_t height, float* __restrict__ rowError) {
    const uint32_t y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= height) return;
    float sum = 0.0f, carry = 0.0f;
    for (uint32_t x = 0; x < width; ++x) {
        const float4 pa = __ldg(a + static_cast<size_t>(y) * width + x);
        const float4 pb = __ldg(b + static_cast<size_t>(y) * width + x);
        const float va[4] = {pa.x, pa.y, pa.z, pa.w}, vb[4] = {pb.x, pb.y, pb.z, pb.w};
        float squared = 0.0f;
        for (int c = 0; c < 4; ++c) {
            const float d = fabsf(va[c] - vb[c]);
            squared += d * d / (vb[c] * vb[c] + 1e-2f);
        }
        kahan_add(sum, carry, squared * 0.25f);
    }
    rowError[y] = sum + carry;
}

__global__ void float_sum_kernel(const float* __restrict__ values, uint32_t count, float* __restrict__ total) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float sum = 0.0f, carry = 0.0f;
    for (uint32_t i = 0; i < count; ++i) kahan_add(sum, carry, values[i]);
    *total = sum + carry;
}

__global__ void __launch_bounds__(kCompareThreads)
count_different_kernel(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint32_t count,
                       unsigned long long* __restrict__ total) {
    uint32_t n = 0;
    for (uint32_t i = blockIdx.x * kCompareThreads + threadIdx.x; i < count; i += gridDim.x * kCompareThreads)
        n += __ldg(a + i) != __ldg(b + i) ? 1u : 0u;
    n = __reduce_add_sync(0xFFFFFFFFu, n);
    if ((threadIdx.x & 31u) == 0 && n != 0) atomicAdd(total, static_cast<unsigned long long>(n));
}

uint32_t grid_for(uint32_t items) {
    return std::max<uint32_t>(1u, std::min<uint32_t>((items + kCompareThreads - 1) / kCompareThreads, 148u * 8u));
}

}  // namespace

// histogram: 256 zeroed words.
cudaError_t launch_compare_images(const float4* a, const float4* b, uint32_t pixels, uint32_t* histogram,
                                  cudaStream_t stream) {
    if (pixels == 0) return cudaSuccess;
    compare_images_kernel<<<grid_for(pixels), kCompareThreads, 0, stream>>>(a, b, pixels, histogram);
    return cudaGetLastError();
}

// histogram: 256 zeroed words; rowError: height floats; total: one float.
cudaError_t launch_compare_hdr(const float4* a, const float4* b, uint32_t width, uint32_t height, uint32_t* histogram,
                               float* rowError, float* total, cudaStream_t stream) {
    const uint32_t pixels = width * height;
    if (pixels == 0) return cudaSuccess;
    hdr_histogram_kernel<<<grid_for(pixels), kCompareThreads, 0, stream>>>(a, b, pixels, histogram);
    hdr_rows_kernel<<<(height + 63) / 64, 64, 0, stream>>>(a, b, width, height, rowError);
    float_sum_kernel<<<1, 32, 0, stream>>>(rowError, height, total);
    return cudaGetLastError();
}

// total: one zeroed 64-bit word.
cudaError_t launch_count_different(const uint32_t* a, const uint32_t* b, uint32_t count, uint64_t* total,
                                   cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    count_different_kernel<<<grid_for(count), kCompareThreads, 0, stream>>>(
        a, b, count, reinterpret_cast<unsigned long long*>(total));
    return cudaGetLastError();
}

}  // namespace lrt
