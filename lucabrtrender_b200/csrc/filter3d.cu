// The Mip-Splatting 3D smoothing filter's per-splat variance (Yu, Chen,
// Huang, Sattler, Geiger, "Mip-Splatting: Alias-free 3D Gaussian Splatting",
// CVPR 2024, section 4.1). The reference has only the screen-space 2D filter
// (shaders/lrt/splat/splat_project.slang:120-137); this is an opt-in
// extension, off unless a cloud carries a filter array (lrt_gpu_splats.filter3d).
//
// The method: a splat's sampling rate under a camera is the number of pixels
// a unit of length covers at its depth, focal / z. Over the cameras that see
// it, the highest rate r bounds the finest detail any of them can resolve,
// and the splat is convolved with an isotropic Gaussian of variance
// coefficient / r^2 (the paper's coefficient is 0.2), which the projection
// folds into the splat's scales and opacity. "Sees" is taken as: centre in
// front of the near plane, projected within the image widened by 15% on each
// side (the band the EWA Jacobian's clamp covers). Splats no camera sees get
// the largest variance of the seen ones.
//
// B200 layout: one thread per splat; every thread of a block reads the same
// camera at the same time (a broadcast), so the cameras stay in L1. A warp
// reduces its lowest positive rate before one atomicMin on its float bits
// (positive floats order as their bit patterns do).
#include "kernels.cuh"
#include "raster_common.cuh"
#include "rast_handle.h"

namespace lrt {
namespace {

constexpr uint32_t kFilterThreads = 256;

__global__ void __launch_bounds__(kFilterThreads)
filter3d_rate_kernel(const float4* __restrict__ positions, uint32_t n, const FrameParams* __restrict__ cams,
                     uint32_t camCount, float* __restrict__ rate, uint32_t* __restrict__ minRateBits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float best = 0.0f;
    if (i < n) {
        const float4 po = __ldg(positions + i);
        const float3 p = make_float3(po.x, po.y, po.z);
        for (uint32_t c = 0; c < camCount; ++c) {
            const FrameParams& f = cams[c];
            const float3 t = to_view(f, p);
            if (!(t.z > f.nearZ)) continue;
            const float invZ = f.ortho != 0 ? 1.0f : 1.0f / t.z;
            const float sx = f.focalX * t.x * invZ + f.centreX;
            const float sy = f.focalY * t.y * invZ + f.centreY;
            const float w = static_cast<float>(f.width), h = static_cast<float>(f.height);
            if (!(sx >= -0.15f * w && sx <= 1.15f * w && sy >= -0.15f * h && sy <= 1.15f * h)) continue;
            const float r = f.focalX * invZ;
            if (r > best) best = r;
        }
        rate[i] = best;
    }
    uint32_t bits = best > 0.0f ? __float_as_uint(best) : 0xFFFFFFFFu;
    bits = __reduce_min_sync(0xFFFFFFFFu, bits);
    if ((threadIdx.x & 31u) == 0 && bits != 0xFFFFFFFFu) atomicMin(minRateBits, bits);
}

__global__ void __launch_bounds__(kFilterThreads)
filter3d_variance_kernel(float* __restrict__ values, uint32_t n, float coefficient,
                         const uint32_t* __restrict__ minRateBits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float r = values[i];
    if (!(r > 0.0f)) {
        const uint32_t bits = *minRateBits;
        if (bits == 0xFFFFFFFFu) {   // no camera sees any splat
            values[i] = 0.0f;
            return;
        }
        r = __uint_as_float(bits);
    }
    values[i] = coefficient / (r * r);
}

}  // namespace
}  // namespace lrt

extern "C" int lrt_rast_filter3d(lrt_rast* r, const lrt_gpu_splats* cloud, const lrt_projection* cameras,
                                 const uint32_t* sizes, uint32_t cameraCount, float coefficient, float* variance,
                                 void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (cloud == nullptr) return fail(r, LRT_INVALID_ARGUMENT, "null cloud");
    if (cloud->count == 0) return LRT_OK;
    if (cloud->positions == nullptr || variance == nullptr) return fail(r, LRT_INVALID_ARGUMENT, "null buffers");
    if (cameraCount > 0 && (cameras == nullptr || sizes == nullptr))
        return fail(r, LRT_INVALID_ARGUMENT, "null cameras");
    if (!(coefficient >= 0.0f)) return fail(r, LRT_INVALID_ARGUMENT, "the coefficient must be >= 0");
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    // Each camera as the renderer's own frame parameters of the cloud with
    // an identity transform: the same float conversions as a frame.
    std::vector<lrt::FrameParams> hostCams(std::max<uint32_t>(cameraCount, 1));
    CloudDesc desc;
    desc.packed = cloud;
    desc.objectToWorld = kIdentity;
    desc.count = cloud->count;
    for (uint32_t c = 0; c < cameraCount; ++c) {
        lrt_render_settings s{};
        s.width = sizes[2 * c];
        s.height = sizes[2 * c + 1];
        if (s.width == 0 || s.height == 0) return fail(r, LRT_INVALID_ARGUMENT, "zero camera size");
        hostCams[c] = frame_params(&cameras[c], &s, desc, 1, 1, 0);
    }
    LRT_CUDA(r, ensure(r->filterCameras, hostCams.size() * sizeof(lrt::FrameParams)), "filter cameras");
    LRT_CUDA(r, ensure(r->filterScratch, 16), "filter scratch");
    if (cameraCount > 0)
        LRT_CUDA(r, cudaMemcpyAsync(r->filterCameras.ptr, hostCams.data(), cameraCount * sizeof(lrt::FrameParams),
                                    cudaMemcpyHostToDevice, stream),
                 "filter cameras");
    uint32_t* minBits = static_cast<uint32_t*>(r->filterScratch.ptr);
    LRT_CUDA(r, cudaMemsetAsync(minBits, 0xFF, 4, stream), "filter scratch");
    const uint32_t n = cloud->count;
    const uint32_t blocks = (n + lrt::kFilterThreads - 1) / lrt::kFilterThreads;
    lrt::filter3d_rate_kernel<<<blocks, lrt::kFilterThreads, 0, stream>>>(
        static_cast<const float4*>(cloud->positions), n, static_cast<const lrt::FrameParams*>(r->filterCameras.ptr),
        cameraCount, variance, minBits);
    LRT_CUDA(r, cudaGetLastError(), "filter rates");
    lrt::filter3d_variance_kernel<<<blocks, lrt::kFilterThreads, 0, stream>>>(variance, n, coefficient, minBits);
    LRT_CUDA(r, cudaGetLastError(), "filter variances");
    LRT_CUDA(r, cudaEventRecord(r->frameDone, stream), "event");
    r->frameDoneSet = true;
    return LRT_OK;
}
