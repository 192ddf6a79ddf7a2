// Stages (d) tile ranges and (e) the front-to-back blend.
//
// Pair word (64 bits, sorted on its key bits only):
//     tile << (24 + slotBits) | depthKey24 << slotBits | slot
// A stable sort of the key bits [slotBits, slotBits + 24 + tileBits) over
// pairs emitted in slot order leaves every tile's pairs in (depth key, slot)
// order -- the order the reference gets from its depth sort followed by a
// stable tile sort (shaders/lrt/splat/frame.slang:17-20,
// modules/render/src/TileRasterizer.cpp:401-457).
#include "kernels.cuh"
#include "raster_common.cuh"

namespace lrt {
namespace {

constexpr uint32_t kBlendThreads = 256;
constexpr uint32_t kBatch = 256;
constexpr uint32_t kWaitLimit = 1u << 22;

// shaders/lrt/splat/splat_ranges.slang:11-25 (after a zeroing memset,
// splat_tiles_clear.slang:8-17). Each thread takes kRangeRun consecutive
// pairs (two 16-byte loads per pair pair) and the one before them.
constexpr uint32_t kRangeRun = 8;
__global__ void ranges_kernel(const unsigned long long* __restrict__ pairs, const uint32_t* __restrict__ dCount,
                              uint32_t cap, uint32_t tileShift, uint2* __restrict__ ranges) {
    const uint32_t n = min(*dCount, cap);
    const uint32_t first = (blockIdx.x * blockDim.x + threadIdx.x) * kRangeRun;
    if (first >= n) return;
    uint32_t prev = first == 0 ? 0xFFFFFFFFu : static_cast<uint32_t>(__ldg(pairs + first - 1) >> tileShift);
    unsigned long long w[kRangeRun];
    if (first + kRangeRun <= n) {
        const ulonglong2* v = reinterpret_cast<const ulonglong2*>(pairs + first);
#pragma unroll
        for (uint32_t k = 0; k < kRangeRun / 2; ++k) {
            const ulonglong2 q = __ldg(v + k);
            w[2 * k] = q.x;
            w[2 * k + 1] = q.y;
        }
    } else {
#pragma unroll
        for (uint32_t k = 0; k < kRangeRun; ++k) w[k] = first + k < n ? __ldg(pairs + first + k) : 0ull;
    }
#pragma unroll
    for (uint32_t k = 0; k < kRangeRun; ++k) {
        const uint32_t i = first + k;
        if (i < n) {
            const uint32_t t = static_cast<uint32_t>(w[k] >> tileShift);
            if (t != prev) {
                ranges[t].x = i;
                if (i > 0) ranges[prev].y = i;
            }
            prev = t;
        }
    }
    // The run's last pair closes its tile when the pair after it (or the end) differs.
    const uint32_t last = min(first + kRangeRun, n) - 1;
    if (last + 1 == n || static_cast<uint32_t>(__ldg(pairs + last + 1) >> tileShift) != prev) ranges[prev].y = last + 1;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// One record (48 bytes, 16-byte aligned at both ends) by the bulk-copy engine.
__device__ __forceinline__ void bulk_copy_record(void* dst, const void* src, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 48, [%2];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bounded wait on a barrier phase; false when the limit passed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t it = 0; it < kWaitLimit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// A box outside which no pixel centre can pass the record's cut, with every
// rounding of the per-pixel test accounted for, so that skipping a record
// for a whole warp never changes a pixel. {power <= k} is an ellipse whose
// bounding half-widths are sqrt(k c / det) and sqrt(k a / det) for the conic
// (a, b, c). The float power of a pixel can fall below the exact one by at
// most ~4u (|a| dx^2 + 2|b| |dx dy| + |c| dy^2) <= 4u kappa power with
// kappa = (|a| + 2|b| + |c|) / lambda_min; det itself carries a relative
// error up to ~4u (|ac| + b^2) / det. delta bounds both with a factor of 8
// to spare; the cut is widened to cutoff / (1 - delta) and the half-widths by
// (1 + delta) plus 1e-3 px. Records where delta is not small are never skipped.
__device__ __forceinline__ float4 cull_box(const ProjRecord& rec) {
    const float a = rec.conic.x, b = rec.conic.y, c = rec.conic.z, cutoff = rec.screen.w;
    const float det = a * c - b * b;
    const float half = 0.5f * (a + c);
    const float root = sqrtf(0.25f * (a - c) * (a - c) + b * b);
    const float lmin = half - root;
    const float kInf = 3.0e38f;
    if (!(det > 0.0f) || !(lmin > 0.0f) || !(cutoff >= 0.0f)) return make_float4(-kInf, kInf, -kInf, kInf);
    const float kappa = (fabsf(a) + 2.0f * fabsf(b) + fabsf(c)) / lmin;
    const float cond = (fabsf(a * c) + b * b) / det;
    const float delta = 32.0f * 5.9604645e-08f * (kappa + cond + 4.0f);
    if (!(delta < 0.25f)) return make_float4(-kInf, kInf, -kInf, kInf);
    const float k = cutoff / (1.0f - delta);
    const float ex = sqrtf(k * c / det) * (1.0f + delta) + 1e-3f;
    const float ey = sqrtf(k * a / det) * (1.0f + delta) + 1e-3f;
    if (!(ex < kInf) || !(ey < kInf)) return make_float4(-kInf, kInf, -kInf, kInf);
    return make_float4(rec.screen.x - ex, rec.screen.x + ex, rec.screen.y - ey, rec.screen.y + ey);
}

// shaders/lrt/splat/splat_blend.slang:23-108 (splat-only entry, :110-114).
// One block per 16x16 tile, one thread per pixel; warp w covers the 8x4
// pixel block ((w & 1) * 8, (w >> 1) * 4). The tile's pairs are read in
// batches of 256: each thread copies one record into shared memory with a
// bulk copy completing on the batch's mbarrier, and batch k+1 is in flight
// while batch k is blended. Each record gets a conservative bounding box
// (cull_box); a warp skips, as a whole, every record whose box misses the
// bounding box of its pixels that are still blending. Each pixel runs the
// reference's loop unchanged over the records it is given, so it stops at
// T < 1e-4 exactly as the reference does; a warp leaves a batch when all its
// pixels have stopped, and the block stops when every pixel has.
// kTrain: also keep, per pixel, the blended colour before linearising with
// the final transmittance, and one past the last pair that contributed --
// what the backward pass re-blends from.
// kComposite: splatBlendComposite (splat_blend.slang:116-120). A disc record
// (colour.w > 0.5) that passes a pixel's cut ends its walk as an opaque hit,
// and with an under layer a pixel stops at the first pair of the tile whose
// depth is at or behind the layer's there -- whether or not that pair touches
// the pixel. Pairs are in depth-key order, not exactly depth order, so that
// first pair is found from a running maximum of the batch's depths (the first
// index where it reaches the layer's depth), not from depth order.
// Returns true when a bounded wait gave up (kErrTimeout is set): the
// barriers' phases are then unknown, so a persistent caller must stop.
template <bool kTrain, bool kComposite = false>
__device__ __forceinline__ bool blend_tile(const BlendParams& bp, uint32_t tile, uint32_t tx, uint32_t ty,
                                           const uint2* __restrict__ ranges,
                                           const unsigned long long* __restrict__ pairs,
                                           const uint32_t* __restrict__ emitSlot,
                                           const ProjRecord* __restrict__ proj, float4* __restrict__ colourOut,
                                           float* __restrict__ depthOut, float4* __restrict__ pixState,
                                           uint32_t* __restrict__ pixLast, uint32_t* __restrict__ err,
                                           ProjRecord (&sRec)[2][kBatch], float4 (&sBox)[kBatch],
                                           uint64_t (&sBar)[2], uint32_t& phase0, uint32_t& phase1,
                                           const float4* __restrict__ underColour = nullptr,
                                           const float* __restrict__ underDepth = nullptr,
                                           float* sZMax = nullptr, float* sWarpMax = nullptr) {
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u, warp = tid >> 5;
    const uint32_t px = tx * kTile + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t py = ty * kTile + (warp >> 1) * 4u + (lane >> 3);
    const bool inside = px < bp.width && py < bp.height;
    const uint2 range = ranges[tile];
    const uint32_t start = range.x, end = range.y;
    const unsigned long long slotMask = (1ull << bp.slotBits) - 1ull;
    const size_t pix = static_cast<size_t>(py) * bp.width + px;
    // Composite state: the under layer's depth here, where the layer stops
    // this pixel's walk (a pair index), and what ended the walk opaquely.
    bool underHit = false;
    float underZ = 0.0f;
    if constexpr (kComposite) {
        if (underColour != nullptr && inside) {
            underZ = underDepth[pix];
            underHit = underZ > 0.0f;
        }
    }
    uint32_t stopAt = 0xFFFFFFFFu;
    bool opaqueHit = false;
    float4 opaque = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float opaqueZ = 0.0f;
    float zCarry = -3.4e38f;   // the largest depth of the tile's earlier batches

    auto issue = [&](uint32_t buf, uint32_t at) {
        const uint32_t cnt = min(kBatch, end - at);
        if (tid == 0) mbar_arrive_expect_tx(&sBar[buf], cnt * static_cast<uint32_t>(sizeof(ProjRecord)));
        if (tid < cnt) {
            uint32_t slot = static_cast<uint32_t>(pairs[at + tid] & slotMask);
            if constexpr (kTrain) {
                if (emitSlot != nullptr) slot = emitSlot[slot];   // the low field is the emit index
            }
            fence_proxy_async_smem();
            bulk_copy_record(&sRec[buf][tid], proj + slot, &sBar[buf]);
        }
    };

    const float pxf = static_cast<float>(px) + 0.5f;
    const float pyf = static_cast<float>(py) + 0.5f;
    float r = 0.0f, g = 0.0f, b = 0.0f;
    float T = 1.0f;
    float depthSum = 0.0f;
    float depthAt = -1.0f;
    bool done = !inside;
    bool gaveUp = false;
    uint32_t last = start;
    if (start < end) issue(0, start);
    uint32_t k = 0;
    for (uint32_t at = start; at < end; at += kBatch, ++k) {
        const uint32_t buf = k & 1u;
        const bool more = at + kBatch < end;
        if (more) issue(buf ^ 1u, at + kBatch);
        const uint32_t parity = buf == 0 ? phase0 : phase1;
        if (!mbar_wait(&sBar[buf], parity)) {
            atomicOr(err, kErrTimeout);
            done = true;
            gaveUp = true;
        }
        if (buf == 0) phase0 ^= 1u; else phase1 ^= 1u;
        const uint32_t cnt = min(kBatch, end - at);
        const ProjRecord* batch = sRec[buf];
        if (tid < cnt) sBox[tid] = cull_box(batch[tid]);
        if constexpr (kComposite) {
            if (underColour != nullptr) {
                // Running maximum of the depths, tile order, across batches.
                float v = tid < cnt ? batch[tid].screen.z : -3.4e38f;
#pragma unroll
                for (uint32_t d = 1; d < 32; d <<= 1) {
                    const float o = __shfl_up_sync(0xFFFFFFFFu, v, d);
                    if (lane >= d) v = fmaxf(v, o);
                }
                if (lane == 31) sWarpMax[warp] = v;
                __syncthreads();
                float prior = zCarry;
                for (uint32_t w = 0; w < warp; ++w) prior = fmaxf(prior, sWarpMax[w]);
                sZMax[tid] = fmaxf(v, prior);
                __syncthreads();
                zCarry = sZMax[cnt - 1];
                if (underHit && stopAt == 0xFFFFFFFFu && zCarry >= underZ) {
                    uint32_t lo = 0, hi = cnt - 1;   // sZMax[hi] >= underZ
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (sZMax[mid] >= underZ) hi = mid; else lo = mid + 1;
                    }
                    stopAt = at + lo;
                }
            }
        }
        __syncthreads();
        // Records in chunks of 32: each lane tests one record's box against the
        // bounding box of this warp's pixels still blending, and the warp then
        // walks the ballot's set bits in record order.
        for (uint32_t c = 0; c < cnt; c += 32) {
            if constexpr (kComposite) {
                if (at + c >= stopAt) done = true;
            }
            const unsigned active = __ballot_sync(0xFFFFFFFFu, !done);
            if (active == 0) break;
            const uint32_t big = 0xFFFFFFFFu;
            const uint32_t x0 = __reduce_min_sync(0xFFFFFFFFu, done ? big : px);
            const uint32_t x1 = __reduce_max_sync(0xFFFFFFFFu, done ? 0u : px);
            const uint32_t y0 = __reduce_min_sync(0xFFFFFFFFu, done ? big : py);
            const uint32_t y1 = __reduce_max_sync(0xFFFFFFFFu, done ? 0u : py);
            const float bx0 = static_cast<float>(x0) + 0.5f, bx1 = static_cast<float>(x1) + 0.5f;
            const float by0 = static_cast<float>(y0) + 0.5f, by1 = static_cast<float>(y1) + 0.5f;
            bool overlap = false;
            if (c + lane < cnt) {
                const float4 box = sBox[c + lane];
                overlap = !(box.x > bx1 || box.y < bx0 || box.z > by1 || box.w < by0);
            }
            uint32_t todo = __ballot_sync(0xFFFFFFFFu, overlap);
            // Straight-line body with one warp-uniform skip: every lane computes
            // the power, lanes still blending that pass the cut are candidates,
            // and the rest of the reference's step runs predicated on a hit.
            while (todo != 0) {
                const uint32_t j = c + static_cast<uint32_t>(__ffs(todo)) - 1u;
                todo &= todo - 1u;
                const float4 screen = batch[j].screen;
                const float4 conic = batch[j].conic;
                const float dx = pxf - screen.x;
                const float dy = pyf - screen.y;
                const float power = splat_power(conic, dx, dy);
                const bool candidate = !done && !(power > screen.w) && (!kComposite || at + j < stopAt);
                if (!__any_sync(0xFFFFFFFFu, candidate)) continue;
                bool blendIt = candidate;
                if constexpr (kComposite) {
                    if (candidate) {
                        const float4 col = batch[j].colour;
                        if (col.w > 0.5f) {   // a disc: opaque, the walk ends here
                            opaqueHit = true;
                            opaque = make_float4(col.x, col.y, col.z, 1.0f);
                            opaqueZ = screen.z;
                            done = true;
                            blendIt = false;
                        }
                    }
                }
                // A candidate's power lies in [0, 9] (the cut is at most 9), so
                // the exponent's argument is in range; others discard it.
                const float alpha = fminf(0.99f, conic.w * lrt_exp_in_range(-0.5f * power));
                if (blendIt && !(alpha < 1.0f / 255.0f)) {
                    const float4 colour = batch[j].colour;
                    const float weight = T * alpha;
                    // rgb += weight colour, depthSum += weight z
                    // (splat_blend.slang:72-74), each one multiply-add.
                    r = __fmaf_rn(weight, colour.x, r);
                    g = __fmaf_rn(weight, colour.y, g);
                    b = __fmaf_rn(weight, colour.z, b);
                    depthSum = __fmaf_rn(weight, screen.z, depthSum);
                    T = T * (1.0f - alpha);
                    if (depthAt < 0.0f && 1.0f - T >= bp.depthThreshold) depthAt = screen.z;
                    if (kTrain) last = at + j + 1;
                    if (T < 1e-4f) done = true;
                }
            }
        }
        if (__syncthreads_and(done ? 1 : 0)) {
            if (more) {
                // Drain the batch already in flight, and count its phase: a
                // persistent block blends its next tile with the same barriers.
                const uint32_t nb = buf ^ 1u;
                if (!mbar_wait(&sBar[nb], nb == 0 ? phase0 : phase1)) {
                    atomicOr(err, kErrTimeout);
                    gaveUp = true;
                }
                if (nb == 0) phase0 ^= 1u; else phase1 ^= 1u;
            }
            break;
        }
    }
    if (!inside) return gaveUp;
    if constexpr (kComposite) {
        if (!opaqueHit && underHit) {
            opaqueHit = true;
            opaque = underColour[pix];
            opaqueZ = underZ;
        }
    }
    const float coverage = 1.0f - T;
    float lr = r, lg = g, lb = b;
    if (bp.linearise != 0 && coverage > 1e-6f) {
        lr = srgb_to_linear(r / coverage) * coverage;
        lg = srgb_to_linear(g / coverage) * coverage;
        lb = srgb_to_linear(b / coverage) * coverage;
    }
    float4 behind = make_float4(bp.bg[0], bp.bg[1], bp.bg[2], bp.bg[3]);
    if (opaqueHit) {
        behind = opaque;
        depthSum = depthSum + T * opaqueZ;
        if (depthAt < 0.0f) depthAt = opaqueZ;
    }
    const float total = opaqueHit ? 1.0f : coverage;
    colourOut[pix] = make_float4(lr + T * behind.x, lg + T * behind.y, lb + T * behind.z, coverage + T * behind.w);
    depthOut[pix] = bp.depthMode == 0 ? (total > 1e-6f ? depthSum / total : 0.0f) : fmaxf(depthAt, 0.0f);
    if (kTrain) {
        pixState[pix] = make_float4(r, g, b, T);
        pixLast[pix] = last;
    }
    return gaveUp;
}


template <bool kTrain>
__global__ void __launch_bounds__(kBlendThreads)
blend_kernel(BlendParams bp, const uint2* __restrict__ ranges, const unsigned long long* __restrict__ pairs,
             const uint32_t* __restrict__ emitSlot,
             const ProjRecord* __restrict__ proj, float4* __restrict__ colourOut, float* __restrict__ depthOut,
             float4* __restrict__ pixState, uint32_t* __restrict__ pixLast, uint32_t* __restrict__ err) {
    __shared__ __align__(128) ProjRecord sRec[2][kBatch];
    __shared__ __align__(16) float4 sBox[kBatch];
    __shared__ __align__(8) uint64_t sBar[2];
    if (threadIdx.x == 0) {
        mbar_init(&sBar[0], 1);
        mbar_init(&sBar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    uint32_t phase0 = 0, phase1 = 0;
    const uint32_t tile = blockIdx.x;
    blend_tile<kTrain>(bp, tile, tile % bp.tilesX, tile / bp.tilesX, ranges, pairs, emitSlot, proj, colourOut, depthOut,
                       pixState, pixLast, err, sRec, sBox, sBar, phase0, phase1);
}

// splatBlendComposite (splat_blend.slang:116-120): discs and an optional
// under layer (colour may be null).
__global__ void __launch_bounds__(kBlendThreads)
blend_composite_kernel(BlendParams bp, const uint2* __restrict__ ranges, const unsigned long long* __restrict__ pairs,
                       const ProjRecord* __restrict__ proj, float4* __restrict__ colourOut,
                       float* __restrict__ depthOut, const float4* __restrict__ underColour,
                       const float* __restrict__ underDepth, uint32_t* __restrict__ err) {
    __shared__ __align__(128) ProjRecord sRec[2][kBatch];
    __shared__ __align__(16) float4 sBox[kBatch];
    __shared__ __align__(8) uint64_t sBar[2];
    __shared__ float sZMax[kBatch];
    __shared__ float sWarpMax[kBlendThreads / 32];
    if (threadIdx.x == 0) {
        mbar_init(&sBar[0], 1);
        mbar_init(&sBar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    uint32_t phase0 = 0, phase1 = 0;
    const uint32_t tile = blockIdx.x;
    blend_tile<false, true>(bp, tile, tile % bp.tilesX, tile / bp.tilesX, ranges, pairs, nullptr, proj, colourOut,
                            depthOut, nullptr, nullptr, err, sRec, sBox, sBar, phase0, phase1, underColour,
                            underDepth, sZMax, sWarpMax);
}

// Many views in one launch: a persistent grid whose blocks take (view, tile)
// work items from a queue in order -- the views' tiles numbered one after
// another, largest views first -- and blend each as blend_kernel does
// (kTrain: as blend_kernel<true>, keeping each view's per-pixel state).
template <bool kTrain>
__global__ void __launch_bounds__(kBlendThreads)
blend_batch_kernel(BlendParams bp, const ViewParams* __restrict__ views, uint32_t viewCount,
                   const uint2* __restrict__ ranges, const unsigned long long* __restrict__ pairs,
                   const ProjRecord* __restrict__ proj, uint32_t totalTiles, uint32_t* __restrict__ queue,
                   uint32_t* __restrict__ err) {
    __shared__ __align__(128) ProjRecord sRec[2][kBatch];
    __shared__ __align__(16) float4 sBox[kBatch];
    __shared__ __align__(8) uint64_t sBar[2];
    __shared__ uint32_t sItem;
    if (threadIdx.x == 0) {
        mbar_init(&sBar[0], 1);
        mbar_init(&sBar[1], 1);
        mbar_fence_init();
    }
    uint32_t phase0 = 0, phase1 = 0;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) sItem = atomicAdd(queue, 1u);
        __syncthreads();
        const uint32_t item = sItem;
        if (item >= totalTiles) break;
        uint32_t lo = 0, hi = viewCount;   // the view whose tiles hold `item`
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (views[mid].tileBase <= item) lo = mid; else hi = mid;
        }
        const ViewParams v = views[lo];
        BlendParams vbp = bp;
        vbp.width = v.width;
        vbp.height = v.height;
        vbp.tilesX = v.tilesX;
        const uint32_t local = item - v.tileBase;
        const bool gaveUp = blend_tile<kTrain>(vbp, item, local % v.tilesX, local / v.tilesX, ranges, pairs, nullptr,
                                               proj + v.recordBase, v.colour, v.depth,
                                               kTrain ? v.pixState : nullptr, kTrain ? v.pixLast : nullptr, err,
                                               sRec, sBox, sBar, phase0, phase1);
        // After a wait gave up the barriers' phases are unknown: take no more
        // items (the frame reports TIMEOUT and its output is undefined).
        if (__syncthreads_or(gaveUp ? 1 : 0)) return;
    }
}

// d/du of the sRGB-to-linear curve (color.slang:7-10): 0 below zero, 1/12.92
// on the linear segment, 2.4/1.055 ((u + 0.055)/1.055)^1.4 above it.
__device__ __forceinline__ float srgb_to_linear_slope(float c) {
    if (!(c > 0.0f)) return 0.0f;
    if (c <= 0.04045f) return 1.0f / 12.92f;
    return 2.4f / 1.055f * lrt_pow((c + 0.055f) / 1.055f, 1.4f);
}

constexpr uint32_t kGrads = 9;   // d/d(centre x, centre y, conic a, b, c, alpha, r, g, b) per pair
constexpr uint32_t kGradStride = 12;   // floats per pair in the partials buffer (three 16-byte vectors)

// Sum of nine values over the warp by recursive halving (a reduce-scatter):
// at each step a lane keeps part of its list, sends the rest to its partner
// and adds what it receives. The list shrinks 9 -> 5 -> 3 -> 2 -> 1 (lists
// padded with zeros where a half is shorter), so 5 + 3 + 2 + 1 shuffles and a
// last butterfly (12 in all) replace 9 x 5 butterflies. Afterwards lanes l
// and l ^ 1 hold the warp's sum of value `idx` (or idx >= 9: nothing).
__device__ __forceinline__ float warp_reduce_scatter9(const float (&v)[9], uint32_t lane, uint32_t& idx) {
    constexpr unsigned kAll = 0xFFFFFFFFu;
    const bool u16 = (lane & 16u) != 0, u8 = (lane & 8u) != 0, u4 = (lane & 4u) != 0, u2 = (lane & 2u) != 0;
    float a[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) {   // [0..4] | [5..8, -]
        const float lo = v[j], hi = j < 4 ? v[5 + j] : 0.0f;
        a[j] = (u16 ? hi : lo) + __shfl_xor_sync(kAll, u16 ? lo : hi, 16);
    }
    float b[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {   // [0, 1, 2] | [3, 4, -]
        const float lo = a[j], hi = j < 2 ? a[3 + j] : 0.0f;
        b[j] = (u8 ? hi : lo) + __shfl_xor_sync(kAll, u8 ? lo : hi, 8);
    }
    float c[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {   // [0, 1] | [2, -]
        const float lo = b[j], hi = j < 1 ? b[2] : 0.0f;
        c[j] = (u4 ? hi : lo) + __shfl_xor_sync(kAll, u4 ? lo : hi, 4);
    }
    const float d = (u2 ? c[1] : c[0]) + __shfl_xor_sync(kAll, u2 ? c[0] : c[1], 2);   // [0] | [1]
    const uint32_t b1 = u2 ? 1u : 0u;
    const uint32_t pos = u8 ? (u4 ? 5u : 3u + b1) : (u4 ? (b1 != 0 ? 5u : 2u) : b1);   // 5: a padding slot
    idx = pos >= (u16 ? 4u : 5u) ? 9u : (u16 ? 5u : 0u) + pos;
    return d + __shfl_xor_sync(kAll, d, 1);
}

// The backward of blend_kernel<true>: per pixel, the reference's loop run
// backwards from the last pair that contributed, rebuilding each pair's
// transmittance from the final one (T_i = T_{i+1} / (1 - alpha_i)) rather
// than storing it, with B the colour behind the pair:
//   dL/dc_i     = dL/drgb * T_i alpha_i
//   dL/dalpha_i = T_i sum_k dL/drgb_k (c_ik - B_k) - dL/dT * T / (1 - alpha_i)
//   B          <- alpha_i c_i + (1 - alpha_i) B
// then through alpha = min(0.99, alpha0 exp(-power / 2)) (no gradient when
// clamped) and power = a dx^2 + 2 b dx dy + c dy^2. A pair's nine values are
// summed over the warp's pixels by shuffles, over the block's warps in
// warp order through shared memory, and written at the pair's emit index: a
// splat's pairs are contiguous there, so a per-splat sum needs no atomics.
// One tile: `item` indexes the ranges (the frame's tile, or a batch's
// (view, tile) item); (tx, ty) is the tile within its view.
__device__ __forceinline__ void blend_backward_tile(const BlendParams& bp, uint32_t item, uint32_t tx, uint32_t ty,
                                                    const uint2* __restrict__ ranges,
                                                    const unsigned long long* __restrict__ pairs,
                                                    const uint32_t* __restrict__ emit,
                                                    const uint32_t* __restrict__ emitSlot,
                                                    const ProjRecord* __restrict__ proj,
                                                    const float4* __restrict__ pixState,
                                                    const uint32_t* __restrict__ pixLast,
                                                    const float4* __restrict__ gradColour,
                                                    float* __restrict__ partials) {
    constexpr uint32_t kB = 128;
    __shared__ __align__(16) ProjRecord sRec[kB];
    __shared__ __align__(16) float4 sBox[kB];
    __shared__ uint32_t sEmit[kB];
    __shared__ float sPart[kBlendThreads / 32][kB][kGrads];
    __shared__ uint32_t sHit[kBlendThreads / 32][kB / 32];   // which sPart slots a warp wrote this batch
    __shared__ uint32_t sMaxLast;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u, warp = tid >> 5;
    const uint32_t px = tx * kTile + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t py = ty * kTile + (warp >> 1) * 4u + (lane >> 3);
    const bool inside = px < bp.width && py < bp.height;
    const uint2 range = ranges[item];
    const uint32_t start = range.x;
    const unsigned long long slotMask = (1ull << bp.slotBits) - 1ull;
    const size_t pix = static_cast<size_t>(py) * bp.width + px;

    uint32_t myLast = start;
    float gr = 0.0f, gg = 0.0f, gb = 0.0f, gT = 0.0f, T = 1.0f;
    if (inside) {
        myLast = pixLast[pix];
        const float4 st = pixState[pix];
        const float4 G = gradColour[pix];
        T = st.w;
        const float cov = 1.0f - T;
        if (bp.linearise != 0 && cov > 1e-6f) {
            const float u0 = st.x / cov, u1 = st.y / cov, u2 = st.z / cov;
            const float d0 = srgb_to_linear_slope(u0), d1 = srgb_to_linear_slope(u1), d2 = srgb_to_linear_slope(u2);
            gr = G.x * d0;
            gg = G.y * d1;
            gb = G.z * d2;
            // out_k = s(u_k) cov + T bg_k with cov = 1 - T; alpha_out = cov + T bg_a
            gT = G.x * (bp.bg[0] - (srgb_to_linear(u0) - d0 * u0)) + G.y * (bp.bg[1] - (srgb_to_linear(u1) - d1 * u1)) +
                 G.z * (bp.bg[2] - (srgb_to_linear(u2) - d2 * u2)) + G.w * (bp.bg[3] - 1.0f);
        } else {
            gr = G.x;
            gg = G.y;
            gb = G.z;
            gT = G.x * bp.bg[0] + G.y * bp.bg[1] + G.z * bp.bg[2] + G.w * (bp.bg[3] - 1.0f);
        }
    }
    const float Tfinal = T;
    const float gTT = -gT * Tfinal;   // the final transmittance's share of every dL/dalpha
    if (tid == 0) sMaxLast = start;
    __syncthreads();
    if (inside) atomicMax(&sMaxLast, myLast);
    __syncthreads();
    const uint32_t maxLast = sMaxLast;
    bool live = inside && myLast > start;
    // Pairs past every pixel's last contributor get zero partials here, so the
    // buffer needs no clearing beforehand.
    for (uint32_t k = maxLast + tid; k < range.y; k += kBlendThreads) {
        const uint32_t e = emitSlot != nullptr ? static_cast<uint32_t>(pairs[k] & slotMask) : emit[k];
        float4* out = reinterpret_cast<float4*>(partials + static_cast<size_t>(e) * kGradStride);
        out[0] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        out[1] = out[0];
        out[2] = out[0];
    }
    float Br = 0.0f, Bg = 0.0f, Bb = 0.0f;
    const float pxf = static_cast<float>(px) + 0.5f;
    const float pyf = static_cast<float>(py) + 0.5f;

    for (uint32_t bEnd = maxLast; bEnd > start;) {
        const uint32_t bStart = bEnd - start > kB ? bEnd - kB : start;
        const uint32_t cnt = bEnd - bStart;
        if (tid < cnt) {
            const uint32_t low = static_cast<uint32_t>(pairs[bStart + tid] & slotMask);
            // The emit index is the word's low field (and the slot comes from
            // the emit-slot map), or it travelled through the sort as a value.
            const uint32_t slot = emitSlot != nullptr ? emitSlot[low] : low;
            sRec[tid] = proj[slot];
            sEmit[tid] = emitSlot != nullptr ? low : emit[bStart + tid];
        }
        if (tid < (kBlendThreads / 32) * (kB / 32)) (&sHit[0][0])[tid] = 0u;
        __syncthreads();
        if (tid < cnt) sBox[tid] = cull_box(sRec[tid]);
        __syncthreads();
        // Records from the back of the batch, 32 at a time.
        for (int c = static_cast<int>((cnt - 1) & ~31u); c >= 0; c -= 32) {
            const unsigned any = __ballot_sync(0xFFFFFFFFu, live);
            if (any == 0) break;
            // Lanes whose pixel stopped before this chunk take no part in it.
            const bool here = live && myLast > bStart + static_cast<uint32_t>(c);
            if (__ballot_sync(0xFFFFFFFFu, here) == 0) continue;
            const uint32_t big = 0xFFFFFFFFu;
            const uint32_t x0 = __reduce_min_sync(0xFFFFFFFFu, here ? px : big);
            const uint32_t x1 = __reduce_max_sync(0xFFFFFFFFu, here ? px : 0u);
            const uint32_t y0 = __reduce_min_sync(0xFFFFFFFFu, here ? py : big);
            const uint32_t y1 = __reduce_max_sync(0xFFFFFFFFu, here ? py : 0u);
            const float bx0 = static_cast<float>(x0) + 0.5f, bx1 = static_cast<float>(x1) + 0.5f;
            const float by0 = static_cast<float>(y0) + 0.5f, by1 = static_cast<float>(y1) + 0.5f;
            bool overlap = false;
            const uint32_t jl = static_cast<uint32_t>(c) + lane;
            if (jl < cnt) {
                const float4 box = sBox[jl];
                overlap = !(box.x > bx1 || box.y < bx0 || box.z > by1 || box.w < by0);
            }
            uint32_t todo = __ballot_sync(0xFFFFFFFFu, overlap);
            uint32_t written = 0;
            while (todo != 0) {
                const uint32_t bit = 31u - static_cast<uint32_t>(__clz(todo));
                todo &= ~(1u << bit);
                const uint32_t j = static_cast<uint32_t>(c) + bit;
                float v[kGrads] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                const float4 screen = sRec[j].screen;
                const float4 conic = sRec[j].conic;
                const float dx = pxf - screen.x;
                const float dy = pyf - screen.y;
                const float power = splat_power(conic, dx, dy);
                const bool candidate = live && bStart + j < myLast && !(power > screen.w);
                if (!__any_sync(0xFFFFFFFFu, candidate)) continue;
                // The forward's alpha decides who contributed, so it is taken
                // from the exact exponential wherever the fast one (relative
                // error below 1e-6 for these arguments) lies within 1e-5 of
                // either threshold; elsewhere both sides of a threshold agree
                // and the fast value serves.
                float e = __expf(-0.5f * power);
                float raw = conic.w * e;
                if (candidate && (fabsf(raw - 1.0f / 255.0f) <= 1e-5f / 255.0f || fabsf(raw - 0.99f) <= 0.99e-5f)) {
                    e = lrt_exp(-0.5f * power);
                    raw = conic.w * e;
                }
                const float alpha = fminf(0.99f, raw);
                const bool hit = candidate && !(alpha < 1.0f / 255.0f);
                const unsigned hits = __ballot_sync(0xFFFFFFFFu, hit);
                if (hits == 0) continue;
                written |= 1u << bit;
                if (hit) {
                    // Gradients are checked against FP64 to a tolerance, not
                    // bit for bit, so this part uses fused multiply-adds.
                    const float4 col = sRec[j].colour;
                    const float oneMinus = 1.0f - alpha;   // in [0.01, 1]
                    float inv;   // 1 / (1 - alpha) to about 1 ulp
                    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(inv) : "f"(oneMinus));
                    const float Ti = T * inv;
                    const float w = Ti * alpha;
                    v[6] = gr * w;
                    v[7] = gg * w;
                    v[8] = gb * w;
                    const float behind =
                        __fmaf_rn(gr, col.x - Br, __fmaf_rn(gg, col.y - Bg, gb * (col.z - Bb)));
                    const float dAlpha = __fmaf_rn(Ti, behind, gTT * inv);
                    Br = __fmaf_rn(alpha, col.x - Br, Br);
                    Bg = __fmaf_rn(alpha, col.y - Bg, Bg);
                    Bb = __fmaf_rn(alpha, col.z - Bb, Bb);
                    T = Ti;
                    if (raw <= 0.99f) {
                        v[5] = dAlpha * e;
                        const float dPower = -0.5f * alpha * dAlpha;
                        const float pdx = dPower * dx, pdy = dPower * dy;
                        v[2] = pdx * dx;
                        v[3] = 2.0f * pdx * dy;
                        v[4] = pdy * dy;
                        v[0] = -2.0f * __fmaf_rn(conic.x, pdx, conic.y * pdy);
                        v[1] = -2.0f * __fmaf_rn(conic.y, pdx, conic.z * pdy);
                    }
                }
                if ((hits & (hits - 1)) == 0) {
                    // one pixel of the warp: its values are the warp's sums
                    if (hit) {
#pragma unroll
                        for (uint32_t k = 0; k < kGrads; ++k) sPart[warp][j][k] = v[k];
                    }
                } else {
                    uint32_t idx;
                    const float sum = warp_reduce_scatter9(v, lane, idx);
                    if ((lane & 1u) == 0 && idx < kGrads) sPart[warp][j][idx] = sum;
                }
            }
            if (lane == 0) sHit[warp][static_cast<uint32_t>(c) >> 5] = written;
        }
        __syncthreads();
        if (tid < cnt) {
            // Warps that wrote nothing for this record are skipped: adding
            // their zeros would not change the sum.
            float sum[kGradStride] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
            for (uint32_t w = 0; w < kBlendThreads / 32; ++w) {
                if ((sHit[w][tid >> 5] >> (tid & 31u)) & 1u) {
#pragma unroll
                    for (uint32_t k = 0; k < kGrads; ++k) sum[k] += sPart[w][tid][k];
                }
            }
            float4* out = reinterpret_cast<float4*>(partials + static_cast<size_t>(sEmit[tid]) * kGradStride);
            out[0] = make_float4(sum[0], sum[1], sum[2], sum[3]);
            out[1] = make_float4(sum[4], sum[5], sum[6], sum[7]);
            out[2] = make_float4(sum[8], 0.0f, 0.0f, 0.0f);
        }
        __syncthreads();
        bEnd = bStart;
    }
}

__global__ void __launch_bounds__(kBlendThreads)
blend_backward_kernel(BlendParams bp, const uint2* __restrict__ ranges, const unsigned long long* __restrict__ pairs,
                      const uint32_t* __restrict__ emit, const uint32_t* __restrict__ emitSlot,
                      const ProjRecord* __restrict__ proj,
                      const float4* __restrict__ pixState, const uint32_t* __restrict__ pixLast,
                      const float4* __restrict__ gradColour, float* __restrict__ partials) {
    const uint32_t tile = blockIdx.x;
    blend_backward_tile(bp, tile, tile % bp.tilesX, tile / bp.tilesX, ranges, pairs, emit, emitSlot, proj, pixState,
                        pixLast, gradColour, partials);
}

// The backward of a training batch: one block per (view, tile) item of the
// chunk, each the tile of blend_backward_kernel in its own view (records at
// the view's base, pixel state and colour gradient from the view's buffers).
__global__ void __launch_bounds__(kBlendThreads)
blend_backward_batch_kernel(BlendParams bp, const ViewParams* __restrict__ views, uint32_t viewCount,
                            const uint2* __restrict__ ranges, const unsigned long long* __restrict__ pairs,
                            const uint32_t* __restrict__ emit, const ProjRecord* __restrict__ proj,
                            float* __restrict__ partials) {
    const uint32_t item = blockIdx.x;
    uint32_t lo = 0, hi = viewCount;   // the view whose tiles hold `item`
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (views[mid].tileBase <= item) lo = mid; else hi = mid;
    }
    const ViewParams v = views[lo];
    BlendParams vbp = bp;
    vbp.width = v.width;
    vbp.height = v.height;
    vbp.tilesX = v.tilesX;
    const uint32_t local = item - v.tileBase;
    blend_backward_tile(vbp, item, local % v.tilesX, local / v.tilesX, ranges, pairs, emit, nullptr,
                        proj + v.recordBase, v.pixState, v.pixLast, v.gradColour, partials);
}

}  // namespace

cudaError_t launch_ranges(const uint64_t* pairs, const uint32_t* dCount, uint32_t cap, uint32_t tileShift,
                          uint2* ranges, uint32_t tiles, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(ranges, 0, sizeof(uint2) * tiles, stream);
    if (e != cudaSuccess || cap == 0) return e;
    const uint32_t threads = (cap + kRangeRun - 1) / kRangeRun;
    ranges_kernel<<<(threads + 255) / 256, 256, 0, stream>>>(reinterpret_cast<const unsigned long long*>(pairs),
                                                             dCount, cap, tileShift, ranges);
    return cudaGetLastError();
}

cudaError_t launch_blend(const BlendParams& bp, const uint2* ranges, const uint64_t* pairs, const ProjRecord* proj,
                         float4* colour, float* depth, uint32_t* err, cudaStream_t stream) {
    const uint32_t tiles = bp.tilesX * bp.tilesY;
    if (tiles == 0) return cudaSuccess;
    blend_kernel<false><<<tiles, kBlendThreads, 0, stream>>>(
        bp, ranges, reinterpret_cast<const unsigned long long*>(pairs), nullptr, proj, colour, depth, nullptr, nullptr,
        err);
    return cudaGetLastError();
}

cudaError_t launch_blend_composite(const BlendParams& bp, const uint2* ranges, const uint64_t* pairs,
                                  const ProjRecord* proj, float4* colour, float* depth, const float4* underColour,
                                  const float* underDepth, uint32_t* err, cudaStream_t stream) {
    const uint32_t tiles = bp.tilesX * bp.tilesY;
    if (tiles == 0) return cudaSuccess;
    blend_composite_kernel<<<tiles, kBlendThreads, 0, stream>>>(
        bp, ranges, reinterpret_cast<const unsigned long long*>(pairs), proj, colour, depth, underColour, underDepth,
        err);
    return cudaGetLastError();
}

cudaError_t launch_blend_batch(const BlendParams& bp, const ViewParams* views, uint32_t viewCount, const uint2* ranges,
                               const uint64_t* pairs, const ProjRecord* proj, uint32_t totalTiles, uint32_t* queue,
                               uint32_t* err, uint32_t blocks, cudaStream_t stream) {
    if (totalTiles == 0) return cudaSuccess;
    blend_batch_kernel<false><<<blocks, kBlendThreads, 0, stream>>>(
        bp, views, viewCount, ranges, reinterpret_cast<const unsigned long long*>(pairs), proj, totalTiles, queue, err);
    return cudaGetLastError();
}

cudaError_t launch_blend_batch_train(const BlendParams& bp, const ViewParams* views, uint32_t viewCount,
                                     const uint2* ranges, const uint64_t* pairs, const ProjRecord* proj,
                                     uint32_t totalTiles, uint32_t* queue, uint32_t* err, uint32_t blocks,
                                     cudaStream_t stream) {
    if (totalTiles == 0) return cudaSuccess;
    blend_batch_kernel<true><<<blocks, kBlendThreads, 0, stream>>>(
        bp, views, viewCount, ranges, reinterpret_cast<const unsigned long long*>(pairs), proj, totalTiles, queue, err);
    return cudaGetLastError();
}

cudaError_t launch_blend_backward_batch(const BlendParams& bp, const ViewParams* views, uint32_t viewCount,
                                        const uint2* ranges, const uint64_t* pairs, const uint32_t* emit,
                                        const ProjRecord* proj, uint32_t totalTiles, float* partials,
                                        cudaStream_t stream) {
    if (totalTiles == 0) return cudaSuccess;
    blend_backward_batch_kernel<<<totalTiles, kBlendThreads, 0, stream>>>(
        bp, views, viewCount, ranges, reinterpret_cast<const unsigned long long*>(pairs), emit, proj, partials);
    return cudaGetLastError();
}

cudaError_t launch_blend_train(const BlendParams& bp, const uint2* ranges, const uint64_t* pairs,
                               const uint32_t* emitSlot, const ProjRecord* proj, float4* colour, float* depth,
                               float4* pixState, uint32_t* pixLast, uint32_t* err, cudaStream_t stream) {
    const uint32_t tiles = bp.tilesX * bp.tilesY;
    if (tiles == 0) return cudaSuccess;
    blend_kernel<true><<<tiles, kBlendThreads, 0, stream>>>(
        bp, ranges, reinterpret_cast<const unsigned long long*>(pairs), emitSlot, proj, colour, depth, pixState,
        pixLast, err);
    return cudaGetLastError();
}

cudaError_t launch_blend_backward(const BlendParams& bp, const uint2* ranges, const uint64_t* pairs,
                                  const uint32_t* emit, const uint32_t* emitSlot, const ProjRecord* proj,
                                  const float4* pixState, const uint32_t* pixLast, const float4* gradColour,
                                  float* partials, cudaStream_t stream) {
    const uint32_t tiles = bp.tilesX * bp.tilesY;
    if (tiles == 0) return cudaSuccess;
    blend_backward_kernel<<<tiles, kBlendThreads, 0, stream>>>(
        bp, ranges, reinterpret_cast<const unsigned long long*>(pairs), emit, emitSlot, proj, pixState, pixLast,
        gradColour, partials);
    return cudaGetLastError();
}

}  // namespace lrt
