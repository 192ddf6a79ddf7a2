// Device-side frame maths shared by the projection, duplication and blend
// kernels. Each function restates the reference's Slang definition cited
// beside it (paths inside the lucabRTrender tree), expression for expression:
// the library is compiled with -fmad=false, so every product and sum rounds
// once, in the order written, exactly as the CPU oracle's does.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lrt_math.cuh"

#include <utility>

namespace lrt {

// Programmatic dependent launch. A kernel launched by launch_chained may
// have its blocks scheduled while the kernel before it on the stream is
// still finishing: chained_entry<true>(), its first statement, waits until
// that kernel has completed and its writes are visible (which also covers
// every kernel before it), then lets the next chained kernel begin launching
// once all of this grid's blocks are running.
//
// Chaining is on only inside a ChainScope that asks for it: the frame entry
// points open one for frames of at least kChainMinPixels, where the overlap
// was measured to pay (1080p: end to end 1.026 -> 0.957 ms a frame). Smaller
// frames are bound by the host's launch work, so they (and the batched
// paths, sorts and everything else) use the ordinary launch.
constexpr uint64_t kChainMinPixels = 1920ull * 1080ull;
inline thread_local bool tChainLaunches = false;
struct ChainScope {
    bool saved;
    explicit ChainScope(bool on) : saved(tChainLaunches) { tChainLaunches = on; }
    ~ChainScope() { tChainLaunches = saved; }
    ChainScope(const ChainScope&) = delete;
    ChainScope& operator=(const ChainScope&) = delete;
};
// Each chained kernel is compiled twice: with the entry (kChained) for
// chained launches, and without it for ordinary ones, since the entry's two
// instructions cost a measurable time in every block even when a kernel is
// not chained (the same 64 frames 1.35 against 1.48 ms a frame).
template <bool kChained>
__device__ __forceinline__ void chained_entry() {
    if constexpr (kChained) {
        asm volatile("griddepcontrol.wait;" ::: "memory");
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    }
}
template <typename... Params, typename... Args>
inline cudaError_t launch_chained(void (*chained)(Params...), void (*plain)(Params...), dim3 grid, dim3 block,
                                  size_t smem, cudaStream_t stream, Args&&... args) {
    if (!tChainLaunches) {
        plain<<<grid, block, smem, stream>>>(std::forward<Args>(args)...);
        return cudaGetLastError();
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr = {};
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, chained, std::forward<Args>(args)...);
}

constexpr uint32_t kTile = 16;   // shaders/lrt/splat/frame.slang:31
// The largest frame side: the projection packs a splat's tile rectangle
// into 16-bit fields (its height into 15), so a side holds at most 2^15 tiles.
constexpr uint32_t kMaxFrameSide = (1u << 15) * kTile;

struct EditParams {   // shaders/lrt/common/edit.slang:23-37
    uint32_t active, shape, mode, invert;
    float centre[3], size[3], tint[3];
    float saturation, brightness, opacity, minOpacity, maxScale;
};

// The projection's per-instance uniforms (frame.slang:33-81 without the
// relight fields).
struct FrameParams {
    uint32_t width, height, tilesX, tilesY;
    float focalX, focalY, centreX, centreY, nearZ, farZ;
    uint32_t ortho, antialias;
    float m[12];      // object -> view, rows of a 3x4
    float eye[3];     // the camera in the cloud's space
    uint32_t count, base, restPerColour, shWords, shLimit;
    uint32_t tileBase;     // added to every tile id (the view's first tile in a batch; 0 for one view)
    uint32_t recordBase;   // the view's first record in a batch (0 for one view)
    uint32_t writeDebug;   // 1: write rects, touched counts and depth keys per slot
    EditParams edit;
};

struct BlendParams {
    uint32_t width, height, tilesX, tilesY;
    uint32_t slotBits, tileShift;
    uint32_t depthMode, linearise;
    float depthThreshold;
    float bg[4];
};

// One view of a batch, as the batched blend reads it.
struct ViewParams {
    uint32_t width, height, tilesX, tileBase;   // tileBase: the view's first tile in the batch
    uint32_t recordBase, reserved0, reserved1, reserved2;
    float4* colour;
    float* depth;
    // Training batches: the view's per-pixel blend state, and the gradient of
    // the loss with respect to its colour image.
    float4* pixState;
    uint32_t* pixLast;
    const float4* gradColour;
};

// frame.slang:85-89: what the projection leaves for the blend.
struct __align__(16) ProjRecord {
    float4 screen;   // centre.xy, view z, cutoff power
    float4 conic;    // a, b, c, alpha
    float4 colour;   // rgb (encoded), 0
};

// splat_blend.slang:58: a Gaussian's power at pixel offset (dx, dy),
// a dx^2 + 2 b dx dy + c dy^2, evaluated left to right with its two sums
// fused into multiply-adds (the contraction a GPU compiler makes of the
// reference's expression). The blend, its backward and the CPU restatement
// all use this form, so they agree on every pair's contribution bit for bit.
__device__ __forceinline__ float splat_power(float4 conic, float dx, float dy) {
    const float t = conic.x * dx * dx;
    const float u = __fmaf_rn(2.0f * conic.y * dx, dy, t);
    return __fmaf_rn(conic.z * dy, dy, u);
}

// Status bits a kernel may raise in the frame's error word.
constexpr uint32_t kErrOverflow = 1u;
constexpr uint32_t kErrTimeout = 2u;
constexpr uint32_t kErrTooManyPairs = 4u;

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

__device__ __forceinline__ float3 to_view(const FrameParams& f, float3 p) {   // frame.slang:91-95
    return make_float3(f.m[0] * p.x + f.m[1] * p.y + f.m[2] * p.z + f.m[3],
                       f.m[4] * p.x + f.m[5] * p.y + f.m[6] * p.z + f.m[7],
                       f.m[8] * p.x + f.m[9] * p.y + f.m[10] * p.z + f.m[11]);
}

__device__ __forceinline__ float cutoff_power(float alpha) {   // frame.slang:105-107
    return fminf(2.0f * lrt_log(fmaxf(255.0f * alpha, 1.0001f)), 9.0f);
}

// frame.slang:113-130 decides a tile by the exact minimum of the quadratic
// form over the box of its pixel centres: 0 when the box holds the centre,
// else the least of four candidates (each edge at its clamped stationary
// point), compared with the cutoff. That minimum is at most the cutoff
// exactly when one candidate is (fminf skips a NaN candidate, and so does the
// <= test), so here the candidates are tested one by one, each computed with
// the reference's expression, and the first within the cutoff answers. The edges nearer the centre go
// first, since a touched tile is usually decided by one of them; an untouched
// tile still evaluates all four.
//
// farGate (far_edge_gate) lets an untouched tile stop after the two nearer
// edges. The power is a quadratic form, q(t p) = t^2 q(p), so the segment
// from any point of the far edges towards the centre leaves the box through
// a nearer edge, where the power is no larger: the exact minimum over the
// box is on the nearer edges. Their two values, each the float power at a
// few ulps from the edge's exact minimiser, exceed that minimum by less than
// a relative 5u kappa (kappa = (|a| + |b| + |c|) / lambda_min bounds the
// terms' sum against the power), and a far candidate's float value falls
// below its exact one by no more. So when both nearer values are above the
// gate, cutoff (1 + 64u kappa), every far candidate is above the cutoff too
// and the answer (false) is the one the four candidates give.
__device__ __forceinline__ bool power_within_over_box(float a, float b, float c, float lox, float loy, float hix,
                                                      float hiy, float cutoff, float farGate = INFINITY) {
    if (lox <= 0.0f && hix >= 0.0f && loy <= 0.0f && hiy >= 0.0f) return 0.0f <= cutoff;
    const bool xNearHi = fabsf(hix) < fabsf(lox), yNearHi = fabsf(hiy) < fabsf(loy);
    bool nearAbove = true;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        {
            const float x = (e == 0) == xNearHi ? hix : lox;
            const float y = c > 1e-12f ? clampf(-b * x / c, loy, hiy) : loy;
            const float q = a * x * x + 2.0f * b * x * y + c * y * y;
            if (q <= cutoff) return true;
            if (e == 0) nearAbove = q > farGate;
        }
        {
            const float y = (e == 0) == yNearHi ? hiy : loy;
            const float x = a > 1e-12f ? clampf(-b * y / a, lox, hix) : lox;
            const float q = a * x * x + 2.0f * b * x * y + c * y * y;
            if (q <= cutoff) return true;
            if (e == 0) nearAbove = nearAbove && q > farGate;
        }
        if (e == 0 && nearAbove) return false;
    }
    return false;
}

// The gate for power_within_over_box: infinite (never used) unless the conic
// is positive definite with kappa <= 1e4 and both stationary points are
// computed (a, c > 1e-12).
__device__ __forceinline__ float far_edge_gate(float a, float b, float c, float cutoff) {
    if (!(a > 1e-12f) || !(c > 1e-12f) || !(cutoff >= 0.0f)) return INFINITY;
    const float lmin = 0.5f * (a + c) - sqrtf(0.25f * (a - c) * (a - c) + b * b);
    if (!(lmin > 0.0f)) return INFINITY;
    const float kappa = (a + fabsf(b) + c) / lmin;
    if (!(kappa <= 1.0e4f)) return INFINITY;
    return cutoff * (1.0f + 64.0f * 5.9604645e-08f * kappa);
}

// frame.slang:133-138: does tile (tx, ty) hold a pixel centre inside the footprint?
__device__ __forceinline__ bool tile_touched(uint32_t width, uint32_t height, float cx, float cy,
                                             float ca, float cb, float cc, float cutoff, uint32_t tx,
                                             uint32_t ty, float farGate = INFINITY) {
    const float firstX = static_cast<float>(tx * kTile) + 0.5f;
    const float firstY = static_cast<float>(ty * kTile) + 0.5f;
    const float lastX = static_cast<float>(min((tx + 1) * kTile, width) - 1) + 0.5f;
    const float lastY = static_cast<float>(min((ty + 1) * kTile, height) - 1) + 0.5f;
    return power_within_over_box(ca, cb, cc, firstX - cx, firstY - cy, lastX - cx, lastY - cy, cutoff, farGate);
}

// shaders/lrt/common/color.slang:7-10
__device__ __forceinline__ float srgb_to_linear(float c) {
    c = fmaxf(c, 0.0f);
    return c <= 0.04045f ? c / 12.92f : lrt_pow((c + 0.055f) / 1.055f, 2.4f);
}


constexpr float kSqrtHalfF = 0.70710678f;

// decodeQuaternion, packing.slang:52-69: the smallest-three word to (x, y, z, w).
__device__ __forceinline__ void decode_rotation_word(uint32_t word, float& x, float& y, float& z, float& w) {
    const uint32_t largest = word & 3u;
    float sx = static_cast<float>((word >> 22) & 1023u);
    float sy = static_cast<float>((word >> 12) & 1023u);
    float sz = static_cast<float>((word >> 2) & 1023u);
    sx = (sx / 1023.0f * 2.0f - 1.0f) * kSqrtHalfF;
    sy = (sy / 1023.0f * 2.0f - 1.0f) * kSqrtHalfF;
    sz = (sz / 1023.0f * 2.0f - 1.0f) * kSqrtHalfF;
    const float rest = sqrtf(fmaxf(0.0f, 1.0f - (sx * sx + sy * sy + sz * sz)));
    x = largest == 0 ? rest : sx;
    y = largest == 1 ? rest : largest == 0 ? sx : sy;
    z = largest == 2 ? rest : largest == 3 ? sz : sy;
    w = largest == 3 ? rest : sz;
}

// packing.slang:26-50: smallest three of the normalised quaternion.
__device__ __forceinline__ uint32_t encode_quaternion(float4 q0) {
    const float l = sqrtf(q0.x * q0.x + q0.y * q0.y + q0.z * q0.z + q0.w * q0.w);
    float q[4] = {q0.x / l, q0.y / l, q0.z / l, q0.w / l};
    uint32_t largest = 0;
    float best = fabsf(q[0]);
    for (uint32_t k = 1; k < 4; ++k) {
        if (fabsf(q[k]) > best) {
            best = fabsf(q[k]);
            largest = k;
        }
    }
    if (q[largest] < 0.0f) {
        for (float& v : q) v = -v;
    }
    uint32_t word = largest;
    uint32_t shift = 22;
    for (uint32_t k = 0; k < 4; ++k) {
        if (k == largest) continue;
        const float unit = fminf(fmaxf(q[k] / kSqrtHalfF * 0.5f + 0.5f, 0.0f), 1.0f);
        word |= static_cast<uint32_t>(roundf(unit * 1023.0f)) << shift;
        shift -= 10;
    }
    return word;
}

__device__ __forceinline__ float half_safe(float v) { return fminf(fmaxf(v, -65000.0f), 65000.0f); }
// a in the low half, b in the high one, each rounded to nearest even. The
// paired conversion is one instruction on the arithmetic pipe (two scalar
// conversions would take the slower conversion unit); a NaN takes the scalar
// path, which gives the quiet NaN 0x7E00 the host restatement gives.
__device__ __forceinline__ uint32_t pack_halves(float a, float b) {
    if (isnan(a) || isnan(b)) return (float_to_half(a) & 0xFFFFu) | ((float_to_half(b) & 0xFFFFu) << 16);
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Asynchronous global -> shared copies (cp.async): a thread issues all of its
// copies before it waits, so many lines are in flight at once.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_all;" ::: "memory");
}

}  // namespace lrt
