// A STAND-IN for the reference's own GPU path, for comparison only: never
// the product, never called by the package.
//
// The reference runs its splat rasteriser as Slang compute kernels compiled
// at run time (no Slang toolchain exists here, so they cannot run). This file
// runs the same frame with the reference's execution structure on the same
// GPU, written in CUDA from its documented stage sequence and launch shapes
// (modules/render/src/TileRasterizer.cpp:188-484, modules/gpu/src/algo/
// RadixSort.cpp:80-157, PrefixSum.cpp:58-88), so that the sm_100a path has
// a GPU figure to be compared against:
//   project      one thread per splat (groups of 256), plain loads, the exact
//                tile count as a double loop over the rectangle;
//   counts       two chunked prefix sums (one thread per chunk for the chunk
//                totals, one thread walking every chunk total, one thread
//                per chunk for the local scan), then a blocking readback of
//                the visible and pair counts;
//   depth sort   compaction of the visible (key, index), then a 24-bit LSD
//                radix sort: per 8-bit pass a per-chunk histogram (one thread
//                per chunk), digit totals (256 threads walking the chunks),
//                digit starts, and a scatter where one thread walks its chunk
//                in order;
//   emit         the counts gathered in depth order, a prefix sum, and one
//                thread per visible splat repeating the tile test to write
//                its (tile, index) pairs;
//   tile sort    the same radix sort on the tile bits, then ranges;
//   blend        one thread per pixel (16x16 groups) walking its tile's pairs
//                with a 48-byte global record read per (pixel, pair).
// The arithmetic is this library's own (the same projection, tile test and
// blend expressions), so the stand-in's image equals the product's; only
// the schedule differs.
#include "../../lucabrtrender_b200/csrc/rast_handle.h"

#include <cuda_runtime.h>

#include <vector>

namespace {

using lrt::FrameParams;
using lrt::ProjRecord;

struct Standin {
    int device = 0;
    DeviceBuffer proj, rects, touched, visible, keys, scanA, scanB, scanC, chunkTotals, vkeys, vidx, vkeysAlt, vidxAlt,
        counts, offsets, ptiles, pidx, ptilesAlt, pidxAlt, hist, ranges;
    cudaEvent_t ev[7] = {};
    uint32_t* host = nullptr;   // pinned readback
};

constexpr uint32_t kGroup = 256;
constexpr uint32_t kChunkGroup = 64;

// chunkFor (RadixSort.h:40-49): a power of two in [256, 4096], aiming at no
// more than 2048 chunks.
uint32_t chunk_for(uint32_t count) {
    uint32_t c = 256;
    while (c < 4096 && (count + c - 1) / c > 2048) c <<= 1;
    return c;
}

// ---- project -----------------------------------------------------------------
__device__ float3 rest_colour(const uint32_t* row, uint32_t degree, float3 dir) {
    constexpr float kC1 = 0.4886025119029199f;
    auto h = [&](uint32_t q) { return (q & 1u) == 0u ? lrt::low_half(row[q >> 1]) : lrt::high_half(row[q >> 1]); };
    float3 r = make_float3(0.0f, 0.0f, 0.0f);
    if (degree == 0) return r;
    const float x = dir.x, y = dir.y, z = dir.z;
    const float s0 = -kC1 * y, s1 = kC1 * z, s2 = kC1 * x;
    r = make_float3(s0 * h(0) + s1 * h(3) - s2 * h(6), s0 * h(1) + s1 * h(4) - s2 * h(7),
                    s0 * h(2) + s1 * h(5) - s2 * h(8));
    if (degree < 2) return r;
    const float xx = x * x, yy = y * y, zz = z * z;
    const float xy = x * y, yz = y * z, xz = x * z;
    {
        const float t[5] = {1.0925484305920792f * xy, -1.0925484305920792f * yz,
                            0.31539156525252005f * (2.0f * zz - xx - yy), -1.0925484305920792f * xz,
                            0.5462742152960396f * (xx - yy)};
        float a[3] = {0.0f, 0.0f, 0.0f};
        for (int c = 0; c < 3; ++c)
            a[c] = t[0] * h(9 + c) + t[1] * h(12 + c) + t[2] * h(15 + c) + t[3] * h(18 + c) + t[4] * h(21 + c);
        r.x = r.x + a[0];
        r.y = r.y + a[1];
        r.z = r.z + a[2];
    }
    if (degree < 3) return r;
    {
        const float t[7] = {-0.5900435899266435f * y * (3.0f * xx - yy), 2.890611442640554f * xy * z,
                            -0.4570457994644658f * y * (4.0f * zz - xx - yy),
                            0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy),
                            -0.4570457994644658f * x * (4.0f * zz - xx - yy), 1.445305721320277f * z * (xx - yy),
                            -0.5900435899266435f * x * (xx - 3.0f * yy)};
        float a[3];
        for (int c = 0; c < 3; ++c)
            a[c] = t[0] * h(24 + c) + t[1] * h(27 + c) + t[2] * h(30 + c) + t[3] * h(33 + c) + t[4] * h(36 + c) +
                   t[5] * h(39 + c) + t[6] * h(42 + c);
        r.x = r.x + a[0];
        r.y = r.y + a[1];
        r.z = r.z + a[2];
    }
    return r;
}

__global__ void __launch_bounds__(kGroup)
project_kernel(FrameParams f, const float4* __restrict__ positions, const uint4* __restrict__ shape,
               const uint32_t* __restrict__ sh, ProjRecord* __restrict__ proj, uint4* __restrict__ rects,
               uint32_t* __restrict__ touchedOut, uint32_t* __restrict__ visibleOut, uint32_t* __restrict__ keysOut) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= f.count) return;
    const float4 po = positions[i];
    const uint4 sw = shape[i];
    const float3 p = make_float3(po.x, po.y, po.z);
    const float3 scale = make_float3(lrt::lrt_exp(lrt::low_half(sw.y)), lrt::lrt_exp(lrt::high_half(sw.y)),
                                     lrt::lrt_exp(lrt::low_half(sw.z)));
    const float3 t = lrt::to_view(f, p);
    ProjRecord rec;
    rec.screen = rec.conic = rec.colour = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    uint4 rect = make_uint4(1, 1, 0, 0);
    uint32_t touched = 0, key = 0x00FFFFFFu;
    bool alive = (t.z > f.nearZ) && !(t.z > f.farZ);
    float cx = 0, cy = 0, ca = 0, cb = 0, cc = 0, alpha = 0, cutoff = 0;
    if (alive) {
        float x, y, z, w;
        lrt::decode_rotation_word(sw.x, x, y, z, w);
        const float r00 = 1.0f - 2.0f * (y * y + z * z), r01 = 2.0f * (x * y - w * z), r02 = 2.0f * (x * z + w * y);
        const float r10 = 2.0f * (x * y + w * z), r11 = 1.0f - 2.0f * (x * x + z * z), r12 = 2.0f * (y * z - w * x);
        const float r20 = 2.0f * (x * z - w * y), r21 = 2.0f * (y * z + w * x), r22 = 1.0f - 2.0f * (x * x + y * y);
        const float m00 = r00 * scale.x, m01 = r01 * scale.y, m02 = r02 * scale.z;
        const float m10 = r10 * scale.x, m11 = r11 * scale.y, m12 = r12 * scale.z;
        const float m20 = r20 * scale.x, m21 = r21 * scale.y, m22 = r22 * scale.z;
        float jx0, jx1, jx2, jy0, jy1, jy2;
        if (f.ortho) {
            jx0 = f.focalX; jx1 = 0.0f; jx2 = 0.0f;
            jy0 = 0.0f; jy1 = f.focalY; jy2 = 0.0f;
            cx = f.focalX * t.x + f.centreX;
            cy = f.focalY * t.y + f.centreY;
        } else {
            const float invZ = 1.0f / t.z;
            cx = f.focalX * t.x * invZ + f.centreX;
            cy = f.focalY * t.y * invZ + f.centreY;
            const float limLoX = (-0.15f * static_cast<float>(f.width) - f.centreX) / f.focalX;
            const float limHiX = (1.15f * static_cast<float>(f.width) - f.centreX) / f.focalX;
            const float limLoY = (-0.15f * static_cast<float>(f.height) - f.centreY) / f.focalY;
            const float limHiY = (1.15f * static_cast<float>(f.height) - f.centreY) / f.focalY;
            const float tx = lrt::clampf(t.x * invZ, limLoX, limHiX) * t.z;
            const float ty = lrt::clampf(t.y * invZ, limLoY, limHiY) * t.z;
            jx0 = f.focalX * invZ; jx1 = 0.0f; jx2 = -f.focalX * tx * invZ * invZ;
            jy0 = 0.0f; jy1 = f.focalY * invZ; jy2 = -f.focalY * ty * invZ * invZ;
        }
        const float tx0 = jx0 * f.m[0] + jx1 * f.m[4] + jx2 * f.m[8];
        const float tx1 = jx0 * f.m[1] + jx1 * f.m[5] + jx2 * f.m[9];
        const float tx2 = jx0 * f.m[2] + jx1 * f.m[6] + jx2 * f.m[10];
        const float ty0 = jy0 * f.m[0] + jy1 * f.m[4] + jy2 * f.m[8];
        const float ty1 = jy0 * f.m[1] + jy1 * f.m[5] + jy2 * f.m[9];
        const float ty2 = jy0 * f.m[2] + jy1 * f.m[6] + jy2 * f.m[10];
        const float ax0 = tx0 * m00 + tx1 * m10 + tx2 * m20;
        const float ax1 = tx0 * m01 + tx1 * m11 + tx2 * m21;
        const float ax2 = tx0 * m02 + tx1 * m12 + tx2 * m22;
        const float ay0 = ty0 * m00 + ty1 * m10 + ty2 * m20;
        const float ay1 = ty0 * m01 + ty1 * m11 + ty2 * m21;
        const float ay2 = ty0 * m02 + ty1 * m12 + ty2 * m22;
        float a = ax0 * ax0 + ax1 * ax1 + ax2 * ax2;
        const float b = ax0 * ay0 + ax1 * ay1 + ax2 * ay2;
        float c = ay0 * ay0 + ay1 * ay1 + ay2 * ay2;
        const float detBefore = a * c - b * b;
        a = a + 0.3f;
        c = c + 0.3f;
        const float det = a * c - b * b;
        alive = det > 1e-12f;
        if (alive) {
            alpha = po.w;
            if (f.antialias != 0) alpha = alpha * sqrtf(fmaxf(detBefore, 0.0f) / det);
            alive = alpha >= 1.0f / 255.0f;
        }
        if (alive) {
            ca = c / det;
            cb = -b / det;
            cc = a / det;
            cutoff = lrt::cutoff_power(alpha);
            const float det2 = ca * cc - cb * cb;
            const float inv = det2 > 1e-20f ? 1.0f / det2 : 0.0f;
            const float ex = sqrtf(fmaxf(cutoff * cc * inv, 0.0f));
            const float ey = sqrtf(fmaxf(cutoff * ca * inv, 0.0f));
            const float x1 = cx - ex, y1 = cy - ey, x2 = cx + ex, y2 = cy + ey;
            if (x2 < 0.0f || y2 < 0.0f || x1 >= static_cast<float>(f.width) || y1 >= static_cast<float>(f.height)) {
                alive = false;
            } else {
                rect = make_uint4(static_cast<uint32_t>(fmaxf(x1, 0.0f)) / lrt::kTile,
                                  static_cast<uint32_t>(fmaxf(y1, 0.0f)) / lrt::kTile,
                                  static_cast<uint32_t>(fminf(x2, static_cast<float>(f.width) - 1.0f)) / lrt::kTile,
                                  static_cast<uint32_t>(fminf(y2, static_cast<float>(f.height) - 1.0f)) / lrt::kTile);
                alive = !(rect.x > rect.z || rect.y > rect.w);
            }
        }
        if (alive) {   // the exact count, tile by tile
            for (uint32_t ty = rect.y; ty <= rect.w; ++ty)
                for (uint32_t tx = rect.x; tx <= rect.z; ++tx)
                    touched += lrt::tile_touched(f.width, f.height, cx, cy, ca, cb, cc, cutoff, tx, ty) ? 1u : 0u;
            alive = touched != 0;
        }
    }
    if (alive) {
        const float3 base = make_float3(lrt::high_half(sw.z), lrt::low_half(sw.w), lrt::high_half(sw.w));
        const uint32_t rpc = f.restPerColour;
        const uint32_t stored = rpc >= 15 ? 3u : rpc >= 8 ? 2u : rpc >= 3 ? 1u : 0u;
        const uint32_t degree = min(stored, f.shLimit);
        float3 restc = make_float3(0.0f, 0.0f, 0.0f);
        if (degree > 0) {
            const float dx = p.x - f.eye[0], dy = p.y - f.eye[1], dz = p.z - f.eye[2];
            const float l = sqrtf(dx * dx + dy * dy + dz * dz);
            restc = rest_colour(sh + static_cast<size_t>(i) * f.shWords, degree, make_float3(dx / l, dy / l, dz / l));
        }
        rec.screen = make_float4(cx, cy, t.z, cutoff);
        rec.conic = make_float4(ca, cb, cc, alpha);
        rec.colour = make_float4(fmaxf(base.x + restc.x, 0.0f), fmaxf(base.y + restc.y, 0.0f),
                                 fmaxf(base.z + restc.z, 0.0f), 0.0f);
        key = lrt::float_bits(t.z) >> 7;
    } else {
        touched = 0;
        rect = make_uint4(1, 1, 0, 0);
    }
    proj[i] = rec;
    rects[i] = rect;
    touchedOut[i] = touched;
    visibleOut[i] = alive ? 1u : 0u;
    keysOut[i] = key;
}

// ---- chunked prefix sum (PrefixSum.cpp:58-88) ---------------------------------
__global__ void chunk_totals_kernel(const uint32_t* __restrict__ in, uint32_t n, uint32_t chunk,
                                    uint32_t* __restrict__ totals) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t first = c * chunk;
    if (first >= n) return;
    uint32_t s = 0;
    for (uint32_t k = first; k < min(n, first + chunk); ++k) s += in[k];
    totals[c] = s;
}

__global__ void chunk_starts_kernel(uint32_t* __restrict__ totals, uint32_t chunks, uint32_t* __restrict__ sum) {
    uint32_t s = 0;
    for (uint32_t c = 0; c < chunks; ++c) {
        const uint32_t v = totals[c];
        totals[c] = s;
        s += v;
    }
    *sum = s;
}

__global__ void chunk_local_kernel(const uint32_t* __restrict__ in, uint32_t n, uint32_t chunk,
                                   const uint32_t* __restrict__ starts, uint32_t* __restrict__ out) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t first = c * chunk;
    if (first >= n) return;
    uint32_t s = starts[c];
    for (uint32_t k = first; k < min(n, first + chunk); ++k) {
        const uint32_t v = in[k];
        out[k] = s;
        s += v;
    }
}

// ---- compaction and gathers -------------------------------------------------------
__global__ void compact_kernel(const uint32_t* __restrict__ visible, const uint32_t* __restrict__ offsets,
                               const uint32_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ vkeys,
                               uint32_t* __restrict__ vidx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || visible[i] == 0) return;
    vkeys[offsets[i]] = keys[i];
    vidx[offsets[i]] = i;
}

__global__ void gather_counts_kernel(const uint32_t* __restrict__ vidx, uint32_t v, const uint32_t* __restrict__ touched,
                                     uint32_t* __restrict__ counts) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < v) counts[k] = touched[vidx[k]];
}

// ---- radix sort (RadixSort.cpp:80-157): per 8-bit pass -----------------------------
__global__ void radix_histogram_kernel(const uint32_t* __restrict__ keys, uint32_t n, uint32_t chunk, uint32_t shift,
                                       uint32_t* __restrict__ hist) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t first = c * chunk;
    if (first >= n) return;
    uint32_t* h = hist + static_cast<size_t>(c) * 256;
    for (uint32_t d = 0; d < 256; ++d) h[d] = 0;
    for (uint32_t k = first; k < min(n, first + chunk); ++k) h[(keys[k] >> shift) & 0xFFu] += 1;
}

// Thread d: the digit's running offsets across the chunks (in place), then
// its total into totals[d].
__global__ void radix_totals_kernel(uint32_t* __restrict__ hist, uint32_t chunks, uint32_t* __restrict__ totals) {
    const uint32_t d = threadIdx.x;
    uint32_t s = 0;
    for (uint32_t c = 0; c < chunks; ++c) {
        const uint32_t v = hist[static_cast<size_t>(c) * 256 + d];
        hist[static_cast<size_t>(c) * 256 + d] = s;
        s += v;
    }
    totals[d] = s;
}

__global__ void radix_starts_kernel(uint32_t* __restrict__ totals) {
    uint32_t s = 0;
    for (uint32_t d = 0; d < 256; ++d) {
        const uint32_t v = totals[d];
        totals[d] = s;
        s += v;
    }
}

__global__ void radix_scatter_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, uint32_t n,
                                     uint32_t chunk, uint32_t shift, uint32_t* __restrict__ hist,
                                     const uint32_t* __restrict__ starts, uint32_t* __restrict__ keysOut,
                                     uint32_t* __restrict__ valsOut) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t first = c * chunk;
    if (first >= n) return;
    uint32_t* h = hist + static_cast<size_t>(c) * 256;
    for (uint32_t k = first; k < min(n, first + chunk); ++k) {
        const uint32_t key = keys[k];
        const uint32_t d = (key >> shift) & 0xFFu;
        const uint32_t at = starts[d] + h[d]++;
        keysOut[at] = key;
        valsOut[at] = vals[k];
    }
}

// ---- emit -------------------------------------------------------------------------
__global__ void __launch_bounds__(kGroup)
emit_kernel(FrameParams f, const uint32_t* __restrict__ vidx, uint32_t v, const uint32_t* __restrict__ offsets,
            const ProjRecord* __restrict__ proj, const uint4* __restrict__ rects, uint32_t* __restrict__ ptiles,
            uint32_t* __restrict__ pidx, uint32_t capacity) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= v) return;
    const uint32_t i = vidx[k];
    const ProjRecord rec = proj[i];
    const uint4 rect = rects[i];
    uint32_t at = offsets[k];
    for (uint32_t ty = rect.y; ty <= rect.w; ++ty)
        for (uint32_t tx = rect.x; tx <= rect.z; ++tx)
            if (lrt::tile_touched(f.width, f.height, rec.screen.x, rec.screen.y, rec.conic.x, rec.conic.y,
                                  rec.conic.z, rec.screen.w, tx, ty)) {
                if (at < capacity) {
                    ptiles[at] = ty * f.tilesX + tx;
                    pidx[at] = i;
                }
                ++at;
            }
}

__global__ void ranges_kernel(const uint32_t* __restrict__ ptiles, uint32_t p, uint2* __restrict__ ranges) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p) return;
    const uint32_t t = ptiles[k];
    if (k == 0 || ptiles[k - 1] != t) ranges[t].x = k;
    if (k + 1 == p || ptiles[k + 1] != t) ranges[t].y = k + 1;
}

// ---- blend: one thread per pixel, a global record read per (pixel, pair) ------------
__global__ void blend_kernel(lrt::BlendParams bp, const uint2* __restrict__ ranges, const uint32_t* __restrict__ pidx,
                             const ProjRecord* __restrict__ proj, float4* __restrict__ colourOut,
                             float* __restrict__ depthOut) {
    const uint32_t px = blockIdx.x * 16 + threadIdx.x, py = blockIdx.y * 16 + threadIdx.y;
    if (px >= bp.width || py >= bp.height) return;
    const uint2 range = ranges[blockIdx.y * bp.tilesX + blockIdx.x];
    const float pxf = static_cast<float>(px) + 0.5f, pyf = static_cast<float>(py) + 0.5f;
    float r = 0.0f, g = 0.0f, b = 0.0f, T = 1.0f, depthSum = 0.0f, depthAt = -1.0f;
    for (uint32_t k = range.x; k < range.y; ++k) {
        const ProjRecord rec = proj[pidx[k]];
        const float dx = pxf - rec.screen.x, dy = pyf - rec.screen.y;
        const float power = lrt::splat_power(rec.conic, dx, dy);
        if (power > rec.screen.w) continue;
        const float alpha = fminf(0.99f, rec.conic.w * lrt::lrt_exp_in_range(-0.5f * power));
        if (alpha < 1.0f / 255.0f) continue;
        const float weight = T * alpha;
        r = __fmaf_rn(weight, rec.colour.x, r);
        g = __fmaf_rn(weight, rec.colour.y, g);
        b = __fmaf_rn(weight, rec.colour.z, b);
        depthSum = __fmaf_rn(weight, rec.screen.z, depthSum);
        T = T * (1.0f - alpha);
        if (depthAt < 0.0f && 1.0f - T >= bp.depthThreshold) depthAt = rec.screen.z;
        if (T < 1e-4f) break;
    }
    const float coverage = 1.0f - T;
    float lr = r, lg = g, lb = b;
    if (bp.linearise != 0 && coverage > 1e-6f) {
        lr = lrt::srgb_to_linear(r / coverage) * coverage;
        lg = lrt::srgb_to_linear(g / coverage) * coverage;
        lb = lrt::srgb_to_linear(b / coverage) * coverage;
    }
    const size_t pix = static_cast<size_t>(py) * bp.width + px;
    colourOut[pix] = make_float4(lr + T * bp.bg[0], lg + T * bp.bg[1], lb + T * bp.bg[2], coverage + T * bp.bg[3]);
    depthOut[pix] = bp.depthMode == 0 ? (coverage > 1e-6f ? depthSum / coverage : 0.0f) : fmaxf(depthAt, 0.0f);
}

uint32_t blocks_for(uint32_t n, uint32_t group) { return std::max(1u, (n + group - 1) / group); }

cudaError_t grow_to(DeviceBuffer& b, size_t bytes);

cudaError_t scan(Standin* h, const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* sum, cudaStream_t st) {
    const uint32_t chunk = chunk_for(n), chunks = std::max(1u, (n + chunk - 1) / chunk);
    cudaError_t e = grow_to(h->chunkTotals, size_t{chunks} * 4);
    if (e != cudaSuccess) return e;
    uint32_t* totals = static_cast<uint32_t*>(h->chunkTotals.ptr);
    chunk_totals_kernel<<<blocks_for(chunks, kChunkGroup), kChunkGroup, 0, st>>>(in, n, chunk, totals);
    chunk_starts_kernel<<<1, 1, 0, st>>>(totals, chunks, sum);
    chunk_local_kernel<<<blocks_for(chunks, kChunkGroup), kChunkGroup, 0, st>>>(in, n, chunk, totals, out);
    return cudaGetLastError();
}

// Sorts (keys, vals) on `bits` key bits; returns whether the result is in the alternate buffers.
cudaError_t radix_sort(Standin* h, uint32_t* keys, uint32_t* vals, uint32_t* keysAlt, uint32_t* valsAlt, uint32_t n,
                       uint32_t bits, bool* inAlt, cudaStream_t st) {
    *inAlt = false;
    if (n == 0) return cudaSuccess;
    const uint32_t chunk = chunk_for(n), chunks = (n + chunk - 1) / chunk;
    cudaError_t e = grow_to(h->hist, (size_t{chunks} + 1) * 256 * 4);
    if (e != cudaSuccess) return e;
    uint32_t* hist = static_cast<uint32_t*>(h->hist.ptr);
    uint32_t* totals = hist + static_cast<size_t>(chunks) * 256;
    for (uint32_t shift = 0; shift < bits; shift += 8) {
        radix_histogram_kernel<<<blocks_for(chunks, kChunkGroup), kChunkGroup, 0, st>>>(keys, n, chunk, shift, hist);
        radix_totals_kernel<<<1, 256, 0, st>>>(hist, chunks, totals);
        radix_starts_kernel<<<1, 1, 0, st>>>(totals);
        radix_scatter_kernel<<<blocks_for(chunks, kChunkGroup), kChunkGroup, 0, st>>>(keys, vals, n, chunk, shift, hist,
                                                                                      totals, keysAlt, valsAlt);
        std::swap(keys, keysAlt);
        std::swap(vals, valsAlt);
        *inAlt = !*inAlt;
    }
    return cudaGetLastError();
}

cudaError_t grow_to(DeviceBuffer& b, size_t bytes) {
    if (b.bytes >= bytes && b.ptr != nullptr) return cudaSuccess;
    size_t want = std::max<size_t>(bytes, 1024);
    if (b.ptr != nullptr) want = std::max(want, b.bytes * 3 / 2);
    return ensure(b, want);
}

}  // namespace

extern "C" {

int standin_create(void** out, int device) {
    if (out == nullptr) return LRT_INVALID_ARGUMENT;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return LRT_DEVICE_FAILURE;
    Standin* h = new Standin;
    h->device = device;
    for (auto& e : h->ev) cudaEventCreate(&e);
    if (cudaMallocHost(&h->host, 64) != cudaSuccess) {
        delete h;
        return LRT_DEVICE_FAILURE;
    }
    *out = h;
    return LRT_OK;
}

void standin_destroy(void* handle) {
    Standin* h = static_cast<Standin*>(handle);
    if (h == nullptr) return;
    for (DeviceBuffer* b : {&h->proj, &h->rects, &h->touched, &h->visible, &h->keys, &h->scanA, &h->scanB, &h->scanC,
                            &h->chunkTotals, &h->vkeys, &h->vidx, &h->vkeysAlt, &h->vidxAlt, &h->counts, &h->offsets,
                            &h->ptiles, &h->pidx, &h->ptilesAlt, &h->pidxAlt, &h->hist, &h->ranges})
        if (b->ptr != nullptr) cudaFree(b->ptr);
    for (auto& e : h->ev) cudaEventDestroy(e);
    cudaFreeHost(h->host);
    delete h;
}

// One frame of one packed cloud; stage_ms: project, counts, depth sort, emit,
// tile sort + ranges, blend (CUDA events). Returns when the frame is done.
int standin_render(void* handle, const lrt_projection* pr, const lrt_gpu_splats* cloud,
                   const lrt_render_settings* s, lrt_targets* targets, double* stageMs, void* streamPtr) {
    Standin* h = static_cast<Standin*>(handle);
    if (h == nullptr || pr == nullptr || cloud == nullptr || s == nullptr || targets == nullptr)
        return LRT_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(streamPtr);
    const uint32_t n = cloud->count;
    const uint32_t tilesX = (s->width + lrt::kTile - 1) / lrt::kTile, tilesY = (s->height + lrt::kTile - 1) / lrt::kTile;
    const uint32_t tiles = tilesX * tilesY;
    CloudDesc desc;
    desc.packed = cloud;
    desc.objectToWorld = kIdentity;
    desc.count = n;
    const FrameParams f = frame_params(pr, s, desc, tilesX, tilesY, 0);
    const size_t nn = std::max<uint32_t>(n, 1);
    for (DeviceBuffer* b : {&h->touched, &h->visible, &h->keys, &h->scanA, &h->scanB, &h->vkeys, &h->vidx,
                            &h->vkeysAlt, &h->vidxAlt, &h->counts, &h->offsets})
        if (grow_to(*b, nn * 4) != cudaSuccess) return LRT_OUT_OF_MEMORY;
    if (grow_to(h->proj, nn * sizeof(ProjRecord)) != cudaSuccess || grow_to(h->rects, nn * 16) != cudaSuccess ||
        grow_to(h->ranges, size_t{tiles} * 8) != cudaSuccess || grow_to(h->scanC, 64) != cudaSuccess)
        return LRT_OUT_OF_MEMORY;
    uint32_t* sums = static_cast<uint32_t*>(h->scanC.ptr);
    auto U = [](DeviceBuffer& b) { return static_cast<uint32_t*>(b.ptr); };

    cudaEventRecord(h->ev[0], st);
    project_kernel<<<blocks_for(n, kGroup), kGroup, 0, st>>>(
        f, static_cast<const float4*>(cloud->positions), static_cast<const uint4*>(cloud->shape),
        static_cast<const uint32_t*>(cloud->sh), static_cast<ProjRecord*>(h->proj.ptr), static_cast<uint4*>(h->rects.ptr),
        U(h->touched), U(h->visible), U(h->keys));
    cudaEventRecord(h->ev[1], st);
    // counts: both scans, then a blocking readback of the two totals
    scan(h, U(h->visible), U(h->scanA), n, sums, st);
    scan(h, U(h->touched), U(h->scanB), n, sums + 1, st);
    cudaMemcpyAsync(h->host, sums, 8, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return LRT_DEVICE_FAILURE;
    const uint32_t visible = h->host[0], pairs = h->host[1];
    cudaEventRecord(h->ev[2], st);
    if (grow_to(h->ptiles, size_t{std::max(pairs, 1u)} * 4) != cudaSuccess ||
        grow_to(h->pidx, size_t{std::max(pairs, 1u)} * 4) != cudaSuccess ||
        grow_to(h->ptilesAlt, size_t{std::max(pairs, 1u)} * 4) != cudaSuccess ||
        grow_to(h->pidxAlt, size_t{std::max(pairs, 1u)} * 4) != cudaSuccess)
        return LRT_OUT_OF_MEMORY;
    // depth sort: compact, then 24 bits
    compact_kernel<<<blocks_for(n, kGroup), kGroup, 0, st>>>(U(h->visible), U(h->scanA), U(h->keys), n, U(h->vkeys),
                                                              U(h->vidx));
    bool alt = false;
    radix_sort(h, U(h->vkeys), U(h->vidx), U(h->vkeysAlt), U(h->vidxAlt), visible, 24, &alt, st);
    const uint32_t* vidx = alt ? U(h->vidxAlt) : U(h->vidx);
    cudaEventRecord(h->ev[3], st);
    // emit in depth order
    gather_counts_kernel<<<blocks_for(visible, kGroup), kGroup, 0, st>>>(vidx, visible, U(h->touched), U(h->counts));
    scan(h, U(h->counts), U(h->offsets), visible, sums + 2, st);
    emit_kernel<<<blocks_for(visible, kGroup), kGroup, 0, st>>>(f, vidx, visible, U(h->offsets),
                                                                static_cast<ProjRecord*>(h->proj.ptr),
                                                                static_cast<uint4*>(h->rects.ptr), U(h->ptiles),
                                                                U(h->pidx), pairs);
    cudaEventRecord(h->ev[4], st);
    // tile sort + ranges
    uint32_t tileBits = 1;
    while ((1u << tileBits) < tiles) ++tileBits;
    bool palt = false;
    radix_sort(h, U(h->ptiles), U(h->pidx), U(h->ptilesAlt), U(h->pidxAlt), pairs, tileBits, &palt, st);
    const uint32_t* ptiles = palt ? U(h->ptilesAlt) : U(h->ptiles);
    const uint32_t* pidx = palt ? U(h->pidxAlt) : U(h->pidx);
    cudaMemsetAsync(h->ranges.ptr, 0, size_t{tiles} * 8, st);
    ranges_kernel<<<blocks_for(pairs, kGroup), kGroup, 0, st>>>(ptiles, pairs, static_cast<uint2*>(h->ranges.ptr));
    cudaEventRecord(h->ev[5], st);
    lrt::BlendParams bp{};
    bp.width = s->width;
    bp.height = s->height;
    bp.tilesX = tilesX;
    bp.tilesY = tilesY;
    bp.depthMode = s->depth_mode;
    bp.linearise = s->linearise ? 1u : 0u;
    bp.depthThreshold = s->depth_threshold;
    for (int k = 0; k < 4; ++k) bp.bg[k] = s->background[k];
    blend_kernel<<<dim3(tilesX, tilesY), dim3(16, 16), 0, st>>>(bp, static_cast<uint2*>(h->ranges.ptr), pidx,
                                                                static_cast<ProjRecord*>(h->proj.ptr),
                                                                static_cast<float4*>(targets->colour),
                                                                static_cast<float*>(targets->depth));
    cudaEventRecord(h->ev[6], st);
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return LRT_DEVICE_FAILURE;
    if (stageMs != nullptr)
        for (int k = 0; k < 6; ++k) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, h->ev[k], h->ev[k + 1]);
            stageMs[k] = ms;
        }
    return LRT_OK;
}

}  // extern "C"
