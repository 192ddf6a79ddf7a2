// Stages (d) tile ranges and (e) the front-to-back blend.
//
// Pair words (64 bits, sorted on their tile bits, or on tile and depth):
//   single frames:  tile << 32 | slot (or emit index), emitted in depth order
//                   and sorted stably on the tile bits -- the reference's
//                   depth sort followed by a stable tile sort
//                   (shaders/lrt/splat/frame.slang:17-20,
//                   modules/render/src/TileRasterizer.cpp:401-457);
//   batched views:  tile << (24 + slotBits) | depthKey24 << slotBits | slot,
//                   emitted in slot order and sorted stably on the key bits.
// Both leave every tile's pairs in (depth key, slot) order. BlendParams
// carries the slot field's width (slotBits) and the tile field's shift.
#include "kernels.cuh"
#include "raster_common.cuh"
#include "blend_common.cuh"

namespace lrt {
namespace {

constexpr uint32_t kBatch = 256;
constexpr uint32_t kWaitLimit = 1u << 22;
// Pixels a thread in the splat blends (the composite blend keeps one).
constexpr uint32_t kBlendPix = 2;

// shaders/lrt/splat/splat_ranges.slang:11-25 (after a zeroing memset,
// splat_tiles_clear.slang:8-17). Each thread takes kRangeRun consecutive
// pairs (two 16-byte loads per pair pair) and the one before them.
constexpr uint32_t kRangeRun = 8;
template <bool kChained>
__global__ void ranges_kernel(const unsigned long long* __restrict__ pairs, const uint32_t* __restrict__ dCount,
                              uint32_t cap, uint32_t tileShift, uint2* __restrict__ ranges) {
    chained_entry<kChained>();
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

// shaders/lrt/splat/splat_blend.slang:23-108 (splat-only entry, :110-114).
// One block per 16x16 tile, kPix pixels a thread (kBlendThreads / kPix
// threads); warp w covers the 8 x 4kPix pixel block ((w & 1) * 8,
// (w >> 1) * 4kPix), a lane's pixels 4 rows apart, so the per-record work a
// warp shares (the walk, the record's loads, the votes) serves kPix pixels a
// lane. The tile's pairs are read in batches of 256 / kPix, one record a
// thread, each copied into shared memory by a bulk copy completing on the
// batch's mbarrier; batch k+1 is in flight while batch k is blended. Each record gets a conservative bounding box
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
template <bool kTrain, bool kComposite = false, uint32_t kPix = 1>
__device__ __forceinline__ bool blend_tile(const BlendParams& bp, uint32_t tile, uint32_t tx, uint32_t ty,
                                           const uint2* __restrict__ ranges,
                                           const unsigned long long* __restrict__ pairs,
                                           const uint32_t* __restrict__ emitSlot,
                                           const ProjRecord* __restrict__ proj, float4* __restrict__ colourOut,
                                           float* __restrict__ depthOut, float4* __restrict__ pixState,
                                           uint32_t* __restrict__ pixLast, uint32_t* __restrict__ err,
                                           ProjRecord (&sRec)[2][kBatch / kPix],
                                           float4 (&sBox)[kBatch / kPix], uint64_t (&sBar)[2], uint32_t& phase0,
                                           uint32_t& phase1, const float4* __restrict__ underColour = nullptr,
                                           const float* __restrict__ underDepth = nullptr,
                                           float* sZMax = nullptr, float* sWarpMax = nullptr) {
    static_assert(!kComposite || kPix == 1, "the composite walk keeps one pixel a thread");
    constexpr uint32_t kThreads = kBlendThreads / kPix;
    constexpr uint32_t kB = kBatch / kPix;   // records a batch: one per thread
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u, warp = tid >> 5;
    // Warp w covers the 8 x 4kPix block ((w & 1) * 8, (w >> 1) * 4kPix); a
    // lane's pixel q sits 4q rows below its first.
    const uint32_t px = tx * kTile + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t py0 = ty * kTile + (warp >> 1) * (4u * kPix) + (lane >> 3);
    const uint2 range = ranges[tile];
    const uint32_t start = range.x, end = range.y;
    const unsigned long long slotMask = (1ull << bp.slotBits) - 1ull;
    const float pxf = static_cast<float>(px) + 0.5f;
    bool inside[kPix], done[kPix];
    float pyf[kPix], r[kPix], g[kPix], b[kPix], T[kPix], depthSum[kPix], depthAt[kPix];
    uint32_t last[kPix];
#pragma unroll
    for (uint32_t q = 0; q < kPix; ++q) {
        const uint32_t py = py0 + 4u * q;
        inside[q] = px < bp.width && py < bp.height;
        done[q] = !inside[q];
        pyf[q] = static_cast<float>(py) + 0.5f;
        r[q] = 0.0f;
        g[q] = 0.0f;
        b[q] = 0.0f;
        T[q] = 1.0f;
        depthSum[q] = 0.0f;
        depthAt[q] = -1.0f;
        last[q] = start;
    }
    // Composite state (one pixel a thread): the under layer's depth here,
    // where the layer stops this pixel's walk (a pair index), and what ended
    // the walk opaquely.
    bool underHit = false;
    float underZ = 0.0f;
    if constexpr (kComposite) {
        if (underColour != nullptr && inside[0]) {
            underZ = underDepth[static_cast<size_t>(py0) * bp.width + px];
            underHit = underZ > 0.0f;
        }
    }
    uint32_t stopAt = 0xFFFFFFFFu;
    bool opaqueHit = false;
    float4 opaque = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float opaqueZ = 0.0f;
    float zCarry = -3.4e38f;   // the largest depth of the tile's earlier batches

    auto issue = [&](uint32_t buf, uint32_t at) {
        const uint32_t cnt = min(kB, end - at);
        if (tid == 0) mbar_arrive_expect_tx(&sBar[buf], cnt * static_cast<uint32_t>(sizeof(ProjRecord)));
        for (uint32_t k = tid; k < cnt; k += kThreads) {
            uint32_t slot = static_cast<uint32_t>(pairs[at + k] & slotMask);
            if constexpr (kTrain) {
                if (emitSlot != nullptr) slot = emitSlot[slot];   // the low field is the emit index
            }
            fence_proxy_async_smem();
            bulk_copy_record(&sRec[buf][k], proj + slot, &sBar[buf]);
        }
    };

    bool gaveUp = false;
    if (start < end) issue(0, start);
    uint32_t k = 0;
    for (uint32_t at = start; at < end; at += kB, ++k) {
        const uint32_t buf = k & 1u;
        const bool more = at + kB < end;
        if (more) issue(buf ^ 1u, at + kB);
        const uint32_t parity = buf == 0 ? phase0 : phase1;
        if (!mbar_wait(&sBar[buf], parity)) {
            atomicOr(err, kErrTimeout);
#pragma unroll
            for (uint32_t q = 0; q < kPix; ++q) done[q] = true;
            gaveUp = true;
        }
        if (buf == 0) phase0 ^= 1u; else phase1 ^= 1u;
        const uint32_t cnt = min(kB, end - at);
        const ProjRecord* batch = sRec[buf];
        for (uint32_t m = tid; m < cnt; m += kThreads) sBox[m] = cull_box(batch[m]);
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
                if (at + c >= stopAt) done[0] = true;
            }
            bool live = false;
            uint32_t yLo = 0xFFFFFFFFu, yHi = 0u;
#pragma unroll
            for (uint32_t q = 0; q < kPix; ++q) {
                if (!done[q]) {
                    live = true;
                    yLo = min(yLo, py0 + 4u * q);
                    yHi = max(yHi, py0 + 4u * q);
                }
            }
            const unsigned active = __ballot_sync(0xFFFFFFFFu, live);
            if (active == 0) break;
            const uint32_t big = 0xFFFFFFFFu;
            const uint32_t x0 = __reduce_min_sync(0xFFFFFFFFu, live ? px : big);
            const uint32_t x1 = __reduce_max_sync(0xFFFFFFFFu, live ? px : 0u);
            const uint32_t y0 = __reduce_min_sync(0xFFFFFFFFu, yLo);
            const uint32_t y1 = __reduce_max_sync(0xFFFFFFFFu, yHi);
            const float bx0 = static_cast<float>(x0) + 0.5f, bx1 = static_cast<float>(x1) + 0.5f;
            const float by0 = static_cast<float>(y0) + 0.5f, by1 = static_cast<float>(y1) + 0.5f;
            bool overlap = false;
            if (c + lane < cnt) {
                const float4 box = sBox[c + lane];
                overlap = !(box.x > bx1 || box.y < bx0 || box.z > by1 || box.w < by0);
            }
            uint32_t todo = __ballot_sync(0xFFFFFFFFu, overlap);
            // Straight-line body with warp-uniform skips: every lane computes
            // the power of each of its pixels, pixels still blending that pass
            // the cut are candidates, and the rest of the reference's step
            // runs predicated on a hit.
            while (todo != 0) {
                const uint32_t j = c + static_cast<uint32_t>(__ffs(todo)) - 1u;
                todo &= todo - 1u;
                const float4 screen = batch[j].screen;
                const float4 conic = batch[j].conic;
                const float dx = pxf - screen.x;
                float power[kPix];
                bool candidate[kPix];
                bool anyCandidate = false;
#pragma unroll
                for (uint32_t q = 0; q < kPix; ++q) {
                    const float dy = pyf[q] - screen.y;
                    power[q] = splat_power(conic, dx, dy);
                    candidate[q] = !done[q] && !(power[q] > screen.w) && (!kComposite || at + j < stopAt);
                    anyCandidate = anyCandidate || candidate[q];
                }
                if (!__any_sync(0xFFFFFFFFu, anyCandidate)) continue;
#pragma unroll
                for (uint32_t q = 0; q < kPix; ++q) {
                    if (kPix > 1 && !__any_sync(0xFFFFFFFFu, candidate[q])) continue;
                    bool blendIt = candidate[q];
                    if constexpr (kComposite) {
                        if (candidate[q]) {
                            const float4 col = batch[j].colour;
                            if (col.w > 0.5f) {   // a disc: opaque, the walk ends here
                                opaqueHit = true;
                                opaque = make_float4(col.x, col.y, col.z, 1.0f);
                                opaqueZ = screen.z;
                                done[q] = true;
                                blendIt = false;
                            }
                        }
                    }
                    // A candidate's power lies in [0, 9] (the cut is at most 9), so
                    // the exponent's argument is in range; others discard it.
                    const float alpha = fminf(0.99f, conic.w * lrt_exp_in_range(-0.5f * power[q]));
                    if (blendIt && !(alpha < 1.0f / 255.0f)) {
                        const float4 colour = batch[j].colour;
                        const float weight = T[q] * alpha;
                        // rgb += weight colour, depthSum += weight z
                        // (splat_blend.slang:72-74), each one multiply-add.
                        r[q] = __fmaf_rn(weight, colour.x, r[q]);
                        g[q] = __fmaf_rn(weight, colour.y, g[q]);
                        b[q] = __fmaf_rn(weight, colour.z, b[q]);
                        depthSum[q] = __fmaf_rn(weight, screen.z, depthSum[q]);
                        T[q] = T[q] * (1.0f - alpha);
                        if (depthAt[q] < 0.0f && 1.0f - T[q] >= bp.depthThreshold) depthAt[q] = screen.z;
                        if (kTrain) last[q] = at + j + 1;
                        if (T[q] < 1e-4f) done[q] = true;
                    }
                }
            }
        }
        bool allDone = true;
#pragma unroll
        for (uint32_t q = 0; q < kPix; ++q) allDone = allDone && done[q];
        if (__syncthreads_and(allDone ? 1 : 0)) {
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
#pragma unroll
    for (uint32_t q = 0; q < kPix; ++q) {
        if (!inside[q]) continue;
        const size_t pix = static_cast<size_t>(py0 + 4u * q) * bp.width + px;
        if constexpr (kComposite) {
            if (!opaqueHit && underHit) {
                opaqueHit = true;
                opaque = underColour[pix];
                opaqueZ = underZ;
            }
        }
        const float coverage = 1.0f - T[q];
        float lr = r[q], lg = g[q], lb = b[q];
        if (bp.linearise != 0 && coverage > 1e-6f) {
            lr = srgb_to_linear(r[q] / coverage) * coverage;
            lg = srgb_to_linear(g[q] / coverage) * coverage;
            lb = srgb_to_linear(b[q] / coverage) * coverage;
        }
        float4 behind = make_float4(bp.bg[0], bp.bg[1], bp.bg[2], bp.bg[3]);
        float dSum = depthSum[q], dAt = depthAt[q];
        if (opaqueHit) {
            behind = opaque;
            dSum = dSum + T[q] * opaqueZ;
            if (dAt < 0.0f) dAt = opaqueZ;
        }
        const float total = opaqueHit ? 1.0f : coverage;
        colourOut[pix] = make_float4(lr + T[q] * behind.x, lg + T[q] * behind.y, lb + T[q] * behind.z,
                                     coverage + T[q] * behind.w);
        depthOut[pix] = bp.depthMode == 0 ? (total > 1e-6f ? dSum / total : 0.0f) : fmaxf(dAt, 0.0f);
        if (kTrain) {
            pixState[pix] = make_float4(r[q], g[q], b[q], T[q]);
            pixLast[pix] = last[q];
        }
    }
    return gaveUp;
}


template <bool kTrain, bool kChained>
__global__ void __launch_bounds__(kBlendThreads / kBlendPix)
blend_kernel(BlendParams bp, const uint2* __restrict__ ranges, const unsigned long long* __restrict__ pairs,
             const uint32_t* __restrict__ emitSlot,
             const ProjRecord* __restrict__ proj, float4* __restrict__ colourOut, float* __restrict__ depthOut,
             float4* __restrict__ pixState, uint32_t* __restrict__ pixLast, uint32_t* __restrict__ err,
             const uint32_t* __restrict__ order) {
    chained_entry<kChained>();
    __shared__ __align__(128) ProjRecord sRec[2][kBatch / kBlendPix];
    __shared__ __align__(16) float4 sBox[kBatch / kBlendPix];
    __shared__ __align__(8) uint64_t sBar[2];
    if (threadIdx.x == 0) {
        mbar_init(&sBar[0], 1);
        mbar_init(&sBar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    uint32_t phase0 = 0, phase1 = 0;
    const uint32_t tile = order != nullptr ? order[blockIdx.x] : blockIdx.x;
    blend_tile<kTrain, false, kBlendPix>(bp, tile, tile % bp.tilesX, tile / bp.tilesX, ranges, pairs, emitSlot, proj,
                                         colourOut, depthOut, pixState, pixLast, err, sRec, sBox, sBar, phase0, phase1);
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
__global__ void __launch_bounds__(kBlendThreads / kBlendPix)
blend_batch_kernel(BlendParams bp, const ViewParams* __restrict__ views, uint32_t viewCount,
                   const uint2* __restrict__ ranges, const unsigned long long* __restrict__ pairs,
                   const ProjRecord* __restrict__ proj, uint32_t totalTiles, uint32_t* __restrict__ queue,
                   uint32_t* __restrict__ err) {
    __shared__ __align__(128) ProjRecord sRec[2][kBatch / kBlendPix];
    __shared__ __align__(16) float4 sBox[kBatch / kBlendPix];
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
        const bool gaveUp = blend_tile<kTrain, false, kBlendPix>(
            vbp, item, local % v.tilesX, local / v.tilesX, ranges, pairs, nullptr, proj + v.recordBase, v.colour,
            v.depth, kTrain ? v.pixState : nullptr, kTrain ? v.pixLast : nullptr, err, sRec, sBox, sBar, phase0,
            phase1);
        // After a wait gave up the barriers' phases are unknown: take no more
        // items (the frame reports TIMEOUT and its output is undefined).
        if (__syncthreads_or(gaveUp ? 1 : 0)) return;
    }
}

}  // namespace

cudaError_t launch_ranges(const uint64_t* pairs, const uint32_t* dCount, uint32_t cap, uint32_t tileShift,
                          uint2* ranges, uint32_t tiles, cudaStream_t stream, bool rangesZeroed) {
    cudaError_t e = rangesZeroed ? cudaSuccess : launch_zero(ranges, sizeof(uint2) * tiles, stream);
    if (e != cudaSuccess || cap == 0) return e;
    const uint32_t threads = (cap + kRangeRun - 1) / kRangeRun;
    return launch_chained(ranges_kernel<true>, ranges_kernel<false>, dim3((threads + 255) / 256), dim3(256), 0, stream,
                          reinterpret_cast<const unsigned long long*>(pairs), dCount, cap, tileShift, ranges);
}

namespace {
template <bool kChained>
__global__ void publish_counters_kernel(const uint32_t* __restrict__ counters, uint32_t* hostMapped) {
    chained_entry<kChained>();
    if (threadIdx.x < 4) hostMapped[threadIdx.x] = counters[threadIdx.x];
    __threadfence_system();
}
}  // namespace

cudaError_t launch_publish_counters(const uint32_t* counters, uint32_t* hostMapped, cudaStream_t stream) {
    return launch_chained(publish_counters_kernel<true>, publish_counters_kernel<false>, dim3(1), dim3(32), 0, stream, counters, hostMapped);
}

namespace {
constexpr uint32_t kOrderThreads = 256;
constexpr uint32_t kOrderBuckets = 16;

__device__ __forceinline__ uint32_t order_bucket(uint32_t work) {   // floor(log2(work + 1)), at most 15
    return min(31u - static_cast<uint32_t>(__clz(work + 1u)), kOrderBuckets - 1u);
}
// A tile's work: its pair count, or (work != null) the given value.
__device__ __forceinline__ uint32_t tile_work(const uint2* __restrict__ ranges, const uint32_t* __restrict__ work,
                                              uint32_t t) {
    if (work != nullptr) return work[t];
    const uint2 r = ranges[t];
    return r.y - r.x;
}

// A block's tiles per bucket: per warp by ballots, then in shared memory.
__device__ __forceinline__ uint32_t order_block_counts(const uint2* __restrict__ ranges,
                                                       const uint32_t* __restrict__ work, uint32_t tiles,
                                                       uint32_t (&sWarp)[kOrderThreads / 32][kOrderBuckets],
                                                       uint32_t& rank) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t t = blockIdx.x * kOrderThreads + threadIdx.x;
    const uint32_t b = t < tiles ? order_bucket(tile_work(ranges, work, t)) : kOrderBuckets;
    rank = 0;
#pragma unroll
    for (uint32_t q = 0; q < kOrderBuckets; ++q) {
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, b == q);
        if (lane == 0) sWarp[warp][q] = static_cast<uint32_t>(__popc(m));
        if (b == q) rank = static_cast<uint32_t>(__popc(m & ((1u << lane) - 1u)));
    }
    __syncthreads();
    return b;
}

template <bool kChained>
__global__ void __launch_bounds__(kOrderThreads) tile_order_count_kernel(const uint2* __restrict__ ranges,
                                                                         const uint32_t* __restrict__ work,
                                                                         uint32_t tiles,
                                                                         uint32_t* __restrict__ blockCounts) {
    chained_entry<kChained>();
    __shared__ uint32_t sWarp[kOrderThreads / 32][kOrderBuckets];
    uint32_t rank;
    order_block_counts(ranges, work, tiles, sWarp, rank);
    if (threadIdx.x < kOrderBuckets) {
        uint32_t n = 0;
        for (uint32_t w = 0; w < kOrderThreads / 32; ++w) n += sWarp[w][threadIdx.x];
        blockCounts[blockIdx.x * kOrderBuckets + threadIdx.x] = n;
    }
}

// The tiles in the order the blend launches them: busiest first, by buckets
// of floor(log2(pairs + 1)), index order within a bucket. Blocks start in
// launch order, so the long tiles start early and the short ones fill in at
// the end. Each block reads every block's counts (from the kernel above):
// the buckets' totals give their bases, the earlier blocks' counts its own
// places in each bucket.
template <bool kChained>
__global__ void __launch_bounds__(kOrderThreads) tile_order_place_kernel(const uint2* __restrict__ ranges,
                                                                         const uint32_t* __restrict__ work,
                                                                         uint32_t tiles,
                                                                         const uint32_t* __restrict__ blockCounts,
                                                                         uint32_t* __restrict__ order) {
    chained_entry<kChained>();
    __shared__ uint32_t sWarp[kOrderThreads / 32][kOrderBuckets];
    __shared__ uint32_t sTotal[kOrderBuckets], sBefore[kOrderBuckets];
    if (threadIdx.x < kOrderBuckets) {
        sTotal[threadIdx.x] = 0;
        sBefore[threadIdx.x] = 0;
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < gridDim.x * kOrderBuckets; k += kOrderThreads) {
        const uint32_t v = blockCounts[k];
        if (v == 0) continue;
        atomicAdd(&sTotal[k % kOrderBuckets], v);
        if (k / kOrderBuckets < blockIdx.x) atomicAdd(&sBefore[k % kOrderBuckets], v);
    }
    uint32_t rank;
    const uint32_t b = order_block_counts(ranges, work, tiles, sWarp, rank);   // (its barrier also ends the sums above)
    if (threadIdx.x < kOrderBuckets) {
        const uint32_t q = threadIdx.x;
        uint32_t run = sBefore[q];
        for (uint32_t h = q + 1; h < kOrderBuckets; ++h) run += sTotal[h];   // the busier buckets come first
        for (uint32_t w = 0; w < kOrderThreads / 32; ++w) {
            const uint32_t n = sWarp[w][q];
            sWarp[w][q] = run;
            run += n;
        }
    }
    __syncthreads();
    const uint32_t t = blockIdx.x * kOrderThreads + threadIdx.x;
    if (t < tiles) order[sWarp[threadIdx.x >> 5][b] + rank] = t;
}
}  // namespace

size_t tile_order_scratch_bytes(uint32_t tiles) {
    return size_t{(tiles + kOrderThreads - 1) / kOrderThreads} * kOrderBuckets * sizeof(uint32_t);
}

cudaError_t launch_tile_order(const uint2* ranges, uint32_t tiles, uint32_t* order, uint32_t* scratch,
                              cudaStream_t stream, const uint32_t* work) {
    if (tiles == 0) return cudaSuccess;
    const uint32_t blocks = (tiles + kOrderThreads - 1) / kOrderThreads;
    cudaError_t e = launch_chained(tile_order_count_kernel<true>, tile_order_count_kernel<false>, dim3(blocks), dim3(kOrderThreads), 0, stream, ranges, work,
                                   tiles, scratch);
    if (e != cudaSuccess) return e;
    return launch_chained(tile_order_place_kernel<true>, tile_order_place_kernel<false>, dim3(blocks), dim3(kOrderThreads), 0, stream, ranges, work, tiles,
                          static_cast<const uint32_t*>(scratch), order);
}

namespace {
// A training frame's tile work for the backward blend: the pairs up to the
// tile's last contributor (the largest of its pixels' saved last indices),
// a warp a tile.
template <bool kChained>
__global__ void __launch_bounds__(256) tile_backward_work_kernel(const uint2* __restrict__ ranges,
                                                                 const uint32_t* __restrict__ pixLast, uint32_t width,
                                                                 uint32_t height, uint32_t tilesX, uint32_t tiles,
                                                                 uint32_t* __restrict__ work) {
    chained_entry<kChained>();
    const uint32_t t = blockIdx.x * 8u + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31u;
    if (t >= tiles) return;
    const uint32_t x0 = (t % tilesX) * kTile, y0 = (t / tilesX) * kTile;
    const uint32_t start = ranges[t].x;
    uint32_t last = start;
#pragma unroll
    for (uint32_t k = 0; k < kTile * kTile / 32; ++k) {
        const uint32_t p = k * 32u + lane;
        const uint32_t px = x0 + (p & (kTile - 1u)), py = y0 + p / kTile;
        if (px < width && py < height) last = max(last, pixLast[static_cast<size_t>(py) * width + px]);
    }
    last = __reduce_max_sync(0xFFFFFFFFu, last);
    if (lane == 0) work[t] = last - start;
}
}  // namespace

cudaError_t launch_tile_backward_order(const uint2* ranges, const uint32_t* pixLast, uint32_t width, uint32_t height,
                                       uint32_t tilesX, uint32_t tiles, uint32_t* order, uint32_t* scratch,
                                       uint32_t* work, cudaStream_t stream) {
    if (tiles == 0) return cudaSuccess;
    cudaError_t e = launch_chained(tile_backward_work_kernel<true>, tile_backward_work_kernel<false>, dim3((tiles + 7) / 8), dim3(256), 0, stream, ranges,
                                   pixLast, width, height, tilesX, tiles, work);
    if (e != cudaSuccess) return e;
    return launch_tile_order(ranges, tiles, order, scratch, stream, work);
}

cudaError_t launch_blend(const BlendParams& bp, const uint2* ranges, const uint64_t* pairs, const ProjRecord* proj,
                         float4* colour, float* depth, uint32_t* err, cudaStream_t stream, const uint32_t* order) {
    const uint32_t tiles = bp.tilesX * bp.tilesY;
    if (tiles == 0) return cudaSuccess;
    return launch_chained(blend_kernel<false, true>, blend_kernel<false, false>, dim3(tiles), dim3(kBlendThreads / kBlendPix), 0, stream, bp, ranges,
                          reinterpret_cast<const unsigned long long*>(pairs), static_cast<const uint32_t*>(nullptr), proj,
                          colour, depth, static_cast<float4*>(nullptr), static_cast<uint32_t*>(nullptr), err, order);
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

// `blocks` counts blocks of kBlendThreads threads; the grid has kBlendPix
// times as many blocks of kBlendThreads / kBlendPix threads.
cudaError_t launch_blend_batch(const BlendParams& bp, const ViewParams* views, uint32_t viewCount, const uint2* ranges,
                               const uint64_t* pairs, const ProjRecord* proj, uint32_t totalTiles, uint32_t* queue,
                               uint32_t* err, uint32_t blocks, cudaStream_t stream) {
    if (totalTiles == 0) return cudaSuccess;
    blend_batch_kernel<false><<<blocks * kBlendPix, kBlendThreads / kBlendPix, 0, stream>>>(
        bp, views, viewCount, ranges, reinterpret_cast<const unsigned long long*>(pairs), proj, totalTiles, queue, err);
    return cudaGetLastError();
}

cudaError_t launch_blend_batch_train(const BlendParams& bp, const ViewParams* views, uint32_t viewCount,
                                     const uint2* ranges, const uint64_t* pairs, const ProjRecord* proj,
                                     uint32_t totalTiles, uint32_t* queue, uint32_t* err, uint32_t blocks,
                                     cudaStream_t stream) {
    if (totalTiles == 0) return cudaSuccess;
    blend_batch_kernel<true><<<blocks * kBlendPix, kBlendThreads / kBlendPix, 0, stream>>>(
        bp, views, viewCount, ranges, reinterpret_cast<const unsigned long long*>(pairs), proj, totalTiles, queue, err);
    return cudaGetLastError();
}

cudaError_t launch_blend_train(const BlendParams& bp, const uint2* ranges, const uint64_t* pairs,
                               const uint32_t* emitSlot, const ProjRecord* proj, float4* colour, float* depth,
                               float4* pixState, uint32_t* pixLast, uint32_t* err, cudaStream_t stream,
                               const uint32_t* order) {
    const uint32_t tiles = bp.tilesX * bp.tilesY;
    if (tiles == 0) return cudaSuccess;
    return launch_chained(blend_kernel<true, true>, blend_kernel<true, false>, dim3(tiles), dim3(kBlendThreads / kBlendPix), 0, stream, bp, ranges,
                          reinterpret_cast<const unsigned long long*>(pairs), emitSlot, proj, colour, depth, pixState,
                          pixLast, err, order);
}

}  // namespace lrt
