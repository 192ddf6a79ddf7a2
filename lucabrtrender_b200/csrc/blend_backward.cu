// The backward of the training blend (blend_kernel<true>): per pixel the
// forward's loop run backwards, gradients per pair summed without atomics.
//
// This file is compiled with fused multiply-add contraction allowed: its
// results are checked against FP64 oracles to a tolerance, not bit for bit,
// and every decision it shares with the forward (the power against the cut,
// alpha against 1/255 and 0.99) is computed by the same explicit
// expressions as there (splat_power's fused multiply-adds, lrt_exp near the
// thresholds), which contraction leaves unchanged.
#include "kernels.cuh"
#include "raster_common.cuh"
#include "blend_common.cuh"

namespace lrt {
namespace {

// d/du of the sRGB-to-linear curve (color.slang:7-10): 0 below zero, 1/12.92
// on the linear segment, 2.4/1.055 ((u + 0.055)/1.055)^1.4 above it.
__device__ __forceinline__ float srgb_to_linear_slope(float c) {
    if (!(c > 0.0f)) return 0.0f;
    if (c <= 0.04045f) return 1.0f / 12.92f;
    return 2.4f / 1.055f * lrt_pow((c + 0.055f) / 1.055f, 1.4f);
}

// Per pair, as written: d/d(centre x, centre y, conic a, b, c, alpha, r, g,
// b). While a batch is summed, slots 0, 1 and 3 hold the sums of pdx, pdy
// and pdx dy (pdx = dL/dpower dx, pdy = dL/dpower dy); the record's conic
// and the factor 2 are applied when the partials are written.
constexpr uint32_t kGrads = 9;
constexpr uint32_t kGradStride = 12;   // floats per pair in the partials buffer (three 16-byte vectors)
constexpr uint32_t kBwdPix = 2;        // pixels a thread

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
// clamped) and power = a dx^2 + 2 b dx dy + c dy^2. kBwdPix pixels a thread
// (warp w covers the 8 x 4kBwdPix block ((w & 1) * 8, (w >> 1) * 4kBwdPix), a
// lane's pixels 4 rows apart): a lane first adds its pixels' nine values, so
// one warp reduction serves 32 kBwdPix pixels. A pair's values are summed over
// the warp by shuffles, over the block's warps in warp order through shared
// memory, and written at the pair's emit index: a splat's pairs are
// contiguous there, so a per-splat sum needs no atomics.
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
    constexpr uint32_t kP = kBwdPix;
    constexpr uint32_t kThreads = kBlendThreads / kP;
    constexpr uint32_t kWarps = kThreads / 32;
    constexpr uint32_t kB = 128;   // records a batch
    __shared__ __align__(16) ProjRecord sRec[kB];
    __shared__ __align__(16) float4 sBox[kB];
    __shared__ uint32_t sEmit[kB];
    __shared__ float sPart[kWarps][kB][kGrads];
    __shared__ uint32_t sHit[kWarps][kB / 32];   // which sPart slots a warp wrote this batch
    __shared__ uint32_t sMaxLast;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u, warp = tid >> 5;
    const uint32_t px = tx * kTile + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t py0 = ty * kTile + (warp >> 1) * (4u * kP) + (lane >> 3);
    const uint2 range = ranges[item];
    const uint32_t start = range.x;
    const unsigned long long slotMask = (1ull << bp.slotBits) - 1ull;
    const float pxf = static_cast<float>(px) + 0.5f;

    uint32_t myLast[kP];
    float pyf[kP], gr[kP], gg[kP], gb[kP], T[kP], gTT[kP], Br[kP], Bg[kP], Bb[kP];
    bool live[kP];
    uint32_t laneMax = start;
#pragma unroll
    for (uint32_t q = 0; q < kP; ++q) {
        const uint32_t py = py0 + 4u * q;
        const bool inside = px < bp.width && py < bp.height;
        pyf[q] = static_cast<float>(py) + 0.5f;
        myLast[q] = start;
        gr[q] = 0.0f;
        gg[q] = 0.0f;
        gb[q] = 0.0f;
        T[q] = 1.0f;
        float gT = 0.0f;
        if (inside) {
            const size_t pix = static_cast<size_t>(py) * bp.width + px;
            myLast[q] = pixLast[pix];
            const float4 st = pixState[pix];
            const float4 G = gradColour[pix];
            T[q] = st.w;
            const float cov = 1.0f - T[q];
            if (bp.linearise != 0 && cov > 1e-6f) {
                const float u0 = st.x / cov, u1 = st.y / cov, u2 = st.z / cov;
                const float d0 = srgb_to_linear_slope(u0), d1 = srgb_to_linear_slope(u1), d2 = srgb_to_linear_slope(u2);
                gr[q] = G.x * d0;
                gg[q] = G.y * d1;
                gb[q] = G.z * d2;
                // out_k = s(u_k) cov + T bg_k with cov = 1 - T; alpha_out = cov + T bg_a
                gT = G.x * (bp.bg[0] - (srgb_to_linear(u0) - d0 * u0)) +
                     G.y * (bp.bg[1] - (srgb_to_linear(u1) - d1 * u1)) +
                     G.z * (bp.bg[2] - (srgb_to_linear(u2) - d2 * u2)) + G.w * (bp.bg[3] - 1.0f);
            } else {
                gr[q] = G.x;
                gg[q] = G.y;
                gb[q] = G.z;
                gT = G.x * bp.bg[0] + G.y * bp.bg[1] + G.z * bp.bg[2] + G.w * (bp.bg[3] - 1.0f);
            }
        }
        gTT[q] = -gT * T[q];   // the final transmittance's share of every dL/dalpha
        Br[q] = 0.0f;
        Bg[q] = 0.0f;
        Bb[q] = 0.0f;
        live[q] = inside && myLast[q] > start;
        laneMax = max(laneMax, myLast[q]);
    }
    if (tid == 0) sMaxLast = start;
    __syncthreads();
    const uint32_t warpMax = __reduce_max_sync(0xFFFFFFFFu, laneMax);
    if (lane == 0) atomicMax(&sMaxLast, warpMax);
    __syncthreads();
    const uint32_t maxLast = sMaxLast;
    // Pairs past every pixel's last contributor get zero partials here, so the
    // buffer needs no clearing beforehand.
    for (uint32_t k = maxLast + tid; k < range.y; k += kThreads) {
        const uint32_t e = emitSlot != nullptr ? static_cast<uint32_t>(pairs[k] & slotMask) : emit[k];
        float4* out = reinterpret_cast<float4*>(partials + static_cast<size_t>(e) * kGradStride);
        out[0] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        out[1] = out[0];
        out[2] = out[0];
    }

    for (uint32_t bEnd = maxLast; bEnd > start;) {
        const uint32_t bStart = bEnd - start > kB ? bEnd - kB : start;
        const uint32_t cnt = bEnd - bStart;
        for (uint32_t m = tid; m < cnt; m += kThreads) {
            const uint32_t low = static_cast<uint32_t>(pairs[bStart + m] & slotMask);
            // The emit index is the word's low field (and the slot comes from
            // the emit-slot map), or it travelled through the sort as a value.
            const uint32_t slot = emitSlot != nullptr ? emitSlot[low] : low;
            sRec[m] = proj[slot];
            sEmit[m] = emitSlot != nullptr ? low : emit[bStart + m];
        }
        if (tid < kWarps * (kB / 32)) (&sHit[0][0])[tid] = 0u;
        __syncthreads();
        for (uint32_t m = tid; m < cnt; m += kThreads) sBox[m] = cull_box(sRec[m]);
        __syncthreads();
        // Records from the back of the batch, 32 at a time.
        for (int c = static_cast<int>((cnt - 1) & ~31u); c >= 0; c -= 32) {
            bool anyLive = false;
#pragma unroll
            for (uint32_t q = 0; q < kP; ++q) anyLive = anyLive || live[q];
            if (__ballot_sync(0xFFFFFFFFu, anyLive) == 0) break;
            // Pixels that stopped before this chunk take no part in it.
            bool here[kP];
            bool hereAny = false;
            uint32_t yLo = 0xFFFFFFFFu, yHi = 0u;
#pragma unroll
            for (uint32_t q = 0; q < kP; ++q) {
                here[q] = live[q] && myLast[q] > bStart + static_cast<uint32_t>(c);
                if (here[q]) {
                    hereAny = true;
                    yLo = min(yLo, py0 + 4u * q);
                    yHi = max(yHi, py0 + 4u * q);
                }
            }
            if (__ballot_sync(0xFFFFFFFFu, hereAny) == 0) continue;
            const uint32_t big = 0xFFFFFFFFu;
            const uint32_t x0 = __reduce_min_sync(0xFFFFFFFFu, hereAny ? px : big);
            const uint32_t x1 = __reduce_max_sync(0xFFFFFFFFu, hereAny ? px : 0u);
            const uint32_t y0 = __reduce_min_sync(0xFFFFFFFFu, yLo);
            const uint32_t y1 = __reduce_max_sync(0xFFFFFFFFu, yHi);
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
                const float4 screen = sRec[j].screen;
                const float4 conic = sRec[j].conic;
                const float dx = pxf - screen.x;
                float dy[kP], power[kP];
                bool candidate[kP];
                bool anyCandidate = false;
#pragma unroll
                for (uint32_t q = 0; q < kP; ++q) {
                    dy[q] = pyf[q] - screen.y;
                    power[q] = splat_power(conic, dx, dy[q]);
                    candidate[q] = live[q] && bStart + j < myLast[q] && !(power[q] > screen.w);
                    anyCandidate = anyCandidate || candidate[q];
                }
                if (!__any_sync(0xFFFFFFFFu, anyCandidate)) continue;
                float v[kGrads] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                bool hitAny = false;
#pragma unroll
                for (uint32_t q = 0; q < kP; ++q) {
                    // The forward's alpha decides who contributed, so it is
                    // taken from the exact exponential wherever the fast one
                    // (relative error below 1e-6 for these arguments) lies
                    // within 1e-5 of either threshold; elsewhere both sides of
                    // a threshold agree and the fast value serves.
                    float e = __expf(-0.5f * power[q]);
                    float raw = conic.w * e;
                    if (candidate[q] &&
                        (fabsf(raw - 1.0f / 255.0f) <= 1e-5f / 255.0f || fabsf(raw - 0.99f) <= 0.99e-5f)) {
                        e = lrt_exp(-0.5f * power[q]);
                        raw = conic.w * e;
                    }
                    const float alpha = fminf(0.99f, raw);
                    const bool hit = candidate[q] && !(alpha < 1.0f / 255.0f);
                    if (hit) {
                        hitAny = true;
                        // Gradients are checked against FP64 to a tolerance, not
                        // bit for bit, so this part uses fused multiply-adds.
                        const float4 col = sRec[j].colour;
                        const float oneMinus = 1.0f - alpha;   // in [0.01, 1]
                        float inv;   // 1 / (1 - alpha) to about 1 ulp
                        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(inv) : "f"(oneMinus));
                        const float Ti = T[q] * inv;
                        const float w = Ti * alpha;
                        v[6] += gr[q] * w;
                        v[7] += gg[q] * w;
                        v[8] += gb[q] * w;
                        const float behind =
                            __fmaf_rn(gr[q], col.x - Br[q], __fmaf_rn(gg[q], col.y - Bg[q], gb[q] * (col.z - Bb[q])));
                        const float dAlpha = __fmaf_rn(Ti, behind, gTT[q] * inv);
                        Br[q] = __fmaf_rn(alpha, col.x - Br[q], Br[q]);
                        Bg[q] = __fmaf_rn(alpha, col.y - Bg[q], Bg[q]);
                        Bb[q] = __fmaf_rn(alpha, col.z - Bb[q], Bb[q]);
                        T[q] = Ti;
                        if (raw <= 0.99f) {
                            // The centre's gradient, -2 (a pdx + b pdy, b pdx + c pdy),
                            // is linear in (pdx, pdy) with the record's conic: the
                            // pixels' pdx and pdy are summed here and the conic
                            // applied once per record when the partials are written
                            // (and the factor 2 of the b term likewise).
                            v[5] += dAlpha * e;
                            const float dPower = -0.5f * alpha * dAlpha;
                            const float pdx = dPower * dx, pdy = dPower * dy[q];
                            v[2] += pdx * dx;
                            v[3] += pdx * dy[q];
                            v[4] += pdy * dy[q];
                            v[0] += pdx;
                            v[1] += pdy;
                        }
                    }
                }
                const unsigned hits = __ballot_sync(0xFFFFFFFFu, hitAny);
                if (hits == 0) continue;
                written |= 1u << bit;
                if ((hits & (hits - 1)) == 0) {
                    // one lane of the warp: its values are the warp's sums
                    if (hitAny) {
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
        for (uint32_t m = tid; m < cnt; m += kThreads) {
            // Warps that wrote nothing for this record are skipped: adding
            // their zeros would not change the sum.
            float sum[kGradStride] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
            for (uint32_t w = 0; w < kWarps; ++w) {
                if ((sHit[w][m >> 5] >> (m & 31u)) & 1u) {
#pragma unroll
                    for (uint32_t k = 0; k < kGrads; ++k) sum[k] += sPart[w][m][k];
                }
            }
            const float4 conic = sRec[m].conic;
            const float gx = -2.0f * __fmaf_rn(conic.x, sum[0], conic.y * sum[1]);
            const float gy = -2.0f * __fmaf_rn(conic.y, sum[0], conic.z * sum[1]);
            float4* out = reinterpret_cast<float4*>(partials + static_cast<size_t>(sEmit[m]) * kGradStride);
            out[0] = make_float4(gx, gy, sum[2], 2.0f * sum[3]);
            out[1] = make_float4(sum[4], sum[5], sum[6], sum[7]);
            out[2] = make_float4(sum[8], 0.0f, 0.0f, 0.0f);
        }
        __syncthreads();
        bEnd = bStart;
    }
}

template <bool kChained>
__global__ void __launch_bounds__(kBlendThreads / kBwdPix)
blend_backward_kernel(BlendParams bp, const uint2* __restrict__ ranges, const unsigned long long* __restrict__ pairs,
                      const uint32_t* __restrict__ emit, const uint32_t* __restrict__ emitSlot,
                      const ProjRecord* __restrict__ proj,
                      const float4* __restrict__ pixState, const uint32_t* __restrict__ pixLast,
                      const float4* __restrict__ gradColour, float* __restrict__ partials,
                      const uint32_t* __restrict__ order) {
    chained_entry<kChained>();
    const uint32_t tile = order != nullptr ? order[blockIdx.x] : blockIdx.x;
    blend_backward_tile(bp, tile, tile % bp.tilesX, tile / bp.tilesX, ranges, pairs, emit, emitSlot, proj, pixState,
                        pixLast, gradColour, partials);
}

// The backward of a training batch: one block per (view, tile) item of the
// chunk, each the tile of blend_backward_kernel in its own view (records at
// the view's base, pixel state and colour gradient from the view's buffers).
__global__ void __launch_bounds__(kBlendThreads / kBwdPix)
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

cudaError_t launch_blend_backward_batch(const BlendParams& bp, const ViewParams* views, uint32_t viewCount,
                                        const uint2* ranges, const uint64_t* pairs, const uint32_t* emit,
                                        const ProjRecord* proj, uint32_t totalTiles, float* partials,
                                        cudaStream_t stream) {
    if (totalTiles == 0) return cudaSuccess;
    blend_backward_batch_kernel<<<totalTiles, kBlendThreads / kBwdPix, 0, stream>>>(
        bp, views, viewCount, ranges, reinterpret_cast<const unsigned long long*>(pairs), emit, proj, partials);
    return cudaGetLastError();
}

cudaError_t launch_blend_backward(const BlendParams& bp, const uint2* ranges, const uint64_t* pairs,
                                  const uint32_t* emit, const uint32_t* emitSlot, const ProjRecord* proj,
                                  const float4* pixState, const uint32_t* pixLast, const float4* gradColour,
                                  float* partials, cudaStream_t stream, const uint32_t* order) {
    const uint32_t tiles = bp.tilesX * bp.tilesY;
    if (tiles == 0) return cudaSuccess;
    return launch_chained(blend_backward_kernel<true>, blend_backward_kernel<false>, dim3(tiles), dim3(kBlendThreads / kBwdPix), 0, stream, bp, ranges,
                          reinterpret_cast<const unsigned long long*>(pairs), emit, emitSlot, proj, pixState, pixLast,
                          gradColour, partials, order);
}

}  // namespace lrt
