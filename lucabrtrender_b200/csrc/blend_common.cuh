// What the forward and backward blends share: the block size and the
// conservative per-record box a warp tests before walking a record.
#pragma once

#include "raster_common.cuh"

namespace lrt {
namespace {

constexpr uint32_t kBlendThreads = 256;

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

}  // namespace
}  // namespace lrt
