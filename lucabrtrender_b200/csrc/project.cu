// Stages (a) and (b): per-splat projection, the touched-tile count, the
// pairs' offsets and the pairs themselves.
//
// Projection restates shaders/lrt/splat/splat_project.slang:39-221 (the splat
// route; relighting is not part of this path): SplatEdit fate, near/far cull,
// 3D covariance from the smallest-three quaternion and f16 log-scales, EWA
// Jacobian clamped to 1.3x the frustum, Mip-Splatting 2D filter with the
// opacity payback, conic and cut-off, tile rectangle, exact touched-tile
// count, view-dependent colour from f16 spherical harmonics up to degree 3,
// and the 24-bit depth key. The pairs are the reference's splat_emit
// (shaders/lrt/splat/splat_emit.slang:17-50).
//
// Two schedules share the projection (project_emit_kernel<Src, kEmit>):
//  - single frames (kEmit false) stop after the records and counts and write
//    each slot's depth word (depth key << 32 | slot) and aux words (its tile
//    mask, or whether a large splat's rows are all single runs); the depth
//    sort orders the words, depth_offsets_kernel gives each slot its first
//    pair in depth order and emit_pairs_kernel writes the pairs
//    (tile << 32 | slot) -- the reference's own two-sort sequence
//    (TileRasterizer.cpp:383-457);
//  - batched views (kEmit true) write (tile | depth key | slot) words in slot
//    order at offsets from a block scan and a decoupled look-back over the
//    frame's partitions, for one sort per chunk of views.
//
// B200 layout: one thread per splat, 256 per block; a block takes the next
// 256 splats by atomic ticket. Positions and shape are read as 16-byte
// vectors. The block's harmonics rows (92 bytes a splat at degree 3; 256 rows
// start on a 16-byte boundary) are staged into shared memory by 16-byte
// cp.async copies issued first, so they land while the geometry runs. The
// exact tile tests of the warp's splats whose rectangles hold at most 128
// tiles run across the warp together, 32 (splat, tile) pairs a step, and each
// such splat keeps a 128-bit mask of its rectangle's tiles in row-major
// order. Larger splats are counted and written a tile row at a time by the
// whole block: a row plan (the ellipse's x-extent in double precision,
// widened by a margin that covers the float test's rounding) gives each row
// a run that is certainly touched and a few columns at its ends that are
// tested exactly. Pairs of masked splats are written by their warp, lanes on
// consecutive pairs, each pair's tile from the mask bit of its rank.
#include "kernels.cuh"
#include "raster_common.cuh"

#include <cuda/atomic>

namespace lrt {
namespace {

constexpr uint32_t kProjectThreads = 256;

struct Fate {
    bool removed, graded;
    float opacity;
};

// shaders/lrt/common/edit.slang:46-75
__device__ __forceinline__ Fate edit_fate(const EditParams& e, float3 p, float opacity, float3 s) {
    Fate f{false, false, opacity};
    if (e.active == 0) return f;
    if (e.minOpacity > 0.0f && opacity < e.minOpacity) {
        f.removed = true;
        return f;
    }
    if (e.maxScale > 0.0f && fmaxf(fmaxf(fabsf(s.x), fabsf(s.y)), fabsf(s.z)) > e.maxScale) {
        f.removed = true;
        return f;
    }
    const float rx = p.x - e.centre[0], ry = p.y - e.centre[1], rz = p.z - e.centre[2];
    bool inside = e.shape == 1 ? rx * rx + ry * ry + rz * rz <= e.size[0] * e.size[0]
                               : (fabsf(rx) <= e.size[0] && fabsf(ry) <= e.size[1] && fabsf(rz) <= e.size[2]);
    if (e.invert != 0) inside = !inside;
    if ((e.mode == 0 && !inside) || (e.mode == 1 && inside)) {
        f.removed = true;
        return f;
    }
    if (inside) {
        f.graded = true;
        f.opacity = opacity * e.opacity;
        f.removed = !(f.opacity >= 1.0f / 255.0f);
    }
    return f;
}

// edit.slang:78-85 (lerp(a, b, t) = a + (b - a) t)
__device__ __forceinline__ float3 edit_grade(const EditParams& e, float3 c0) {
    const float cx = c0.x * e.tint[0] * e.brightness;
    const float cy = c0.y * e.tint[1] * e.brightness;
    const float cz = c0.z * e.tint[2] * e.brightness;
    const float luma = cx * 0.2126f + cy * 0.7152f + cz * 0.0722f;
    return make_float3(fmaxf(luma + (cx - luma) * e.saturation, 0.0f),
                       fmaxf(luma + (cy - luma) * e.saturation, 0.0f),
                       fmaxf(luma + (cz - luma) * e.saturation, 0.0f));
}

// shaders/lrt/common/sh.slang:8-51, over one staged row of f16 pairs.
__device__ __forceinline__ float half_at(const uint32_t* row, uint32_t index) {
    const uint32_t w = row[index >> 1];
    return (index & 1u) == 0u ? low_half(w) : high_half(w);
}

struct Basis {
    float x, y, z;
};
template <uint32_t kOff>
__device__ __forceinline__ Basis basis_at(const uint32_t* row, uint32_t k) {
    return {half_at(row, kOff + k * 3), half_at(row, kOff + k * 3 + 1), half_at(row, kOff + k * 3 + 2)};
}

// The rest coefficients start kOff halves into the row: 0 in the packed
// layout, 3 (after the DC triple) in the training layout.
template <uint32_t kOff>
__device__ __forceinline__ float3 evaluate_rest(const uint32_t* row, uint32_t degree, float3 dir) {
    constexpr float kC1 = 0.4886025119029199f;
    constexpr float kC2_0 = 1.0925484305920792f, kC2_1 = -1.0925484305920792f, kC2_2 = 0.31539156525252005f,
                    kC2_3 = -1.0925484305920792f, kC2_4 = 0.5462742152960396f;
    constexpr float kC3_0 = -0.5900435899266435f, kC3_1 = 2.890611442640554f, kC3_2 = -0.4570457994644658f,
                    kC3_3 = 0.3731763325901154f, kC3_4 = -0.4570457994644658f, kC3_5 = 1.445305721320277f,
                    kC3_6 = -0.5900435899266435f;
    auto basis = [&](uint32_t k) { return basis_at<kOff>(row, k); };
    if (degree == 0) return make_float3(0.0f, 0.0f, 0.0f);
    const float x = dir.x, y = dir.y, z = dir.z;
    const float s0 = -kC1 * y, s1 = kC1 * z, s2 = kC1 * x;
    const Basis b0 = basis(0), b1 = basis(1), b2 = basis(2);
    float3 r = make_float3(s0 * b0.x + s1 * b1.x - s2 * b2.x, s0 * b0.y + s1 * b1.y - s2 * b2.y,
                           s0 * b0.z + s1 * b1.z - s2 * b2.z);
    if (degree < 2) return r;
    const float xx = x * x, yy = y * y, zz = z * z;
    const float xy = x * y, yz = y * z, xz = x * z;
    {
        const float t0 = kC2_0 * xy, t1 = kC2_1 * yz, t2 = kC2_2 * (2.0f * zz - xx - yy), t3 = kC2_3 * xz,
                    t4 = kC2_4 * (xx - yy);
        const Basis b3 = basis(3), b4 = basis(4), b5 = basis(5), b6 = basis(6),
                    b7 = basis(7);
        r.x = r.x + (t0 * b3.x + t1 * b4.x + t2 * b5.x + t3 * b6.x + t4 * b7.x);
        r.y = r.y + (t0 * b3.y + t1 * b4.y + t2 * b5.y + t3 * b6.y + t4 * b7.y);
        r.z = r.z + (t0 * b3.z + t1 * b4.z + t2 * b5.z + t3 * b6.z + t4 * b7.z);
    }
    if (degree < 3) return r;
    {
        const float t0 = kC3_0 * y * (3.0f * xx - yy), t1 = kC3_1 * xy * z,
                    t2 = kC3_2 * y * (4.0f * zz - xx - yy),
                    t3 = kC3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy),
                    t4 = kC3_4 * x * (4.0f * zz - xx - yy), t5 = kC3_5 * z * (xx - yy),
                    t6 = kC3_6 * x * (xx - 3.0f * yy);
        const Basis b8 = basis(8), b9 = basis(9), b10 = basis(10), b11 = basis(11),
                    b12 = basis(12), b13 = basis(13), b14 = basis(14);
        r.x = r.x + (t0 * b8.x + t1 * b9.x + t2 * b10.x + t3 * b11.x + t4 * b12.x + t5 * b13.x + t6 * b14.x);
        r.y = r.y + (t0 * b8.y + t1 * b9.y + t2 * b10.y + t3 * b11.y + t4 * b12.y + t5 * b13.y + t6 * b14.y);
        r.z = r.z + (t0 * b8.z + t1 * b9.z + t2 * b10.z + t3 * b11.z + t4 * b12.z + t5 * b13.z + t6 * b14.z);
    }
    return r;
}

// Where a splat's parameters come from.
//
// PackedSource: the GpuSplats layout (positions float4, shape uint32x4, sh
// f16 pairs), decoded as splat_project.slang does.
// RawSource: the differentiable parameters -- means float3, log-scales
// float3, quaternions (w, x, y, z) float4 normalised here, opacity logits,
// SH fp16 [16][3] per splat (DC first). Scale is exp(log-scale), opacity
// sigmoid(logit) = 1 / (1 + exp(-logit)) and the base colour 0.5 + SH0 * DC,
// the same arithmetic the packing applies, without its quantisation.
struct PackedSource {
    const float4* positions;
    const uint4* shape;
    const uint32_t* sh;
    const float* filter3d;   // optional: the 3D filter's variance per splat
    static constexpr bool kDisc = false;
    static constexpr uint32_t kRestOffset = 0;
    struct Loaded {
        uint4 sw;
    };
    __device__ __forceinline__ void load(uint32_t i, Loaded& l, float3& p, float& opacity, float3& scale) const {
        const float4 po = __ldg(positions + i);
        l.sw = __ldg(shape + i);
        p = make_float3(po.x, po.y, po.z);
        opacity = po.w;
        scale = make_float3(lrt_exp(low_half(l.sw.y)), lrt_exp(high_half(l.sw.y)), lrt_exp(low_half(l.sw.z)));
        if (filter3d != nullptr) apply_filter3d(__ldg(filter3d + i), scale, opacity);
    }
    // The Mip-Splatting 3D filter (Yu et al., CVPR 2024, section 4.1): the
    // splat convolved with an isotropic Gaussian of variance v keeps its
    // rotation, takes the scales sqrt(s^2 + v) and pays the spread-out
    // energy back in opacity, sqrt(prod s^2 / prod (s^2 + v)).
    __device__ __forceinline__ static void apply_filter3d(float v, float3& s, float& opacity) {
        const float qx = s.x * s.x, qy = s.y * s.y, qz = s.z * s.z;
        const float fx = qx + v, fy = qy + v, fz = qz + v;
        const float before = qx * qy * qz;
        const float after = fx * fy * fz;
        opacity = opacity * sqrtf(before / after);
        s = make_float3(sqrtf(fx), sqrtf(fy), sqrtf(fz));
    }
    // decodeQuaternion, packing.slang:52-69
    __device__ __forceinline__ void rotation(const Loaded& l, float& x, float& y, float& z, float& w) const {
        const uint32_t word = l.sw.x;
        const uint32_t largest = word & 3u;
        float sx = static_cast<float>((word >> 22) & 1023u);
        float sy = static_cast<float>((word >> 12) & 1023u);
        float sz = static_cast<float>((word >> 2) & 1023u);
        sx = (sx / 1023.0f * 2.0f - 1.0f) * 0.70710678f;
        sy = (sy / 1023.0f * 2.0f - 1.0f) * 0.70710678f;
        sz = (sz / 1023.0f * 2.0f - 1.0f) * 0.70710678f;
        const float rest = sqrtf(fmaxf(0.0f, 1.0f - (sx * sx + sy * sy + sz * sz)));
        x = largest == 0 ? rest : sx;
        y = largest == 1 ? rest : largest == 0 ? sx : sy;
        z = largest == 2 ? rest : largest == 3 ? sz : sy;
        w = largest == 3 ? rest : sz;
    }
    __device__ __forceinline__ float3 base(const Loaded& l, const uint32_t*) const {
        return make_float3(high_half(l.sw.z), low_half(l.sw.w), high_half(l.sw.w));
    }
};

struct RawSource {
    const float* means;
    const float* logScales;
    const float* quats;
    const float* logits;
    const uint32_t* sh;
    static constexpr bool kDisc = false;
    static constexpr uint32_t kRestOffset = 3;
    struct Loaded {
        float qw, qx, qy, qz;
    };
    __device__ __forceinline__ void load(uint32_t i, Loaded& l, float3& p, float& opacity, float3& scale) const {
        p = make_float3(__ldg(means + 3 * i), __ldg(means + 3 * i + 1), __ldg(means + 3 * i + 2));
        opacity = 1.0f / (1.0f + lrt_exp(-__ldg(logits + i)));
        scale = make_float3(lrt_exp(__ldg(logScales + 3 * i)), lrt_exp(__ldg(logScales + 3 * i + 1)),
                            lrt_exp(__ldg(logScales + 3 * i + 2)));
        const float4 q = __ldg(reinterpret_cast<const float4*>(quats) + i);
        l.qw = q.x;
        l.qx = q.y;
        l.qy = q.z;
        l.qz = q.w;
    }
    __device__ __forceinline__ void rotation(const Loaded& l, float& x, float& y, float& z, float& w) const {
        const float len = sqrtf(l.qw * l.qw + l.qx * l.qx + l.qy * l.qy + l.qz * l.qz);
        if (len > 0.0f) {
            x = l.qx / len;
            y = l.qy / len;
            z = l.qz / len;
            w = l.qw / len;
        } else {
            x = 0.0f;
            y = 0.0f;
            z = 0.0f;
            w = 1.0f;
        }
    }
    __device__ __forceinline__ float3 base(const Loaded&, const uint32_t* row) const {
        constexpr float kSH0 = 0.28209479177387814f;
        return make_float3(0.5f + kSH0 * half_at(row, 0), 0.5f + kSH0 * half_at(row, 1), 0.5f + kSH0 * half_at(row, 2));
    }
};

// PointSource: a point cloud drawn as opaque discs in the same sort as the
// splats (shaders/lrt/splat/points_project.slang:35-86): positions float4,
// colours two words of fp16 halves per point, and the instance's style.
struct PointSource {
    const float4* positions;
    const uint2* colours;
    const uint32_t* sh;   // none: points carry no harmonics
    uint32_t sizeMode;    // 0 world units, 1 pixels
    float size;           // diameter
    uint32_t constantColour;
    float rgb[3];
    static constexpr bool kDisc = true;
    static constexpr uint32_t kRestOffset = 0;
    struct Loaded {};
    // pointRadius, shaders/lrt/points/point_frame.slang:38-44
    __device__ __forceinline__ float radius(const FrameParams& f, float viewZ) const {
        const float r = sizeMode == 1 ? size * 0.5f
                                      : (f.ortho != 0 ? size * 0.5f * f.focalX : size * 0.5f * f.focalX / viewZ);
        return fmaxf(r, 0.5f);
    }
    __device__ __forceinline__ float3 colour(uint32_t i) const {
        if (constantColour != 0) return make_float3(rgb[0], rgb[1], rgb[2]);
        const uint2 w = __ldg(colours + i);
        return make_float3(low_half(w.x), high_half(w.x), low_half(w.y));
    }
};

// Extra outputs of the training forward: each slot's first pair index, and a
// way back from each sorted pair to its emit index. Either the emit index
// rides through the sort as the pair's value (`values`), or it is the pair
// word's low field and `emitSlot` maps it to the slot (`emitSlot`).
struct TrainOutputs {
    uint32_t* offsets;
    uint32_t* values;
    uint32_t* emitSlot;
};

// Splats of up to kWarpArea tiles have their tiles tested by their warp (32
// (splat, tile) pairs a step) and keep a 128-bit tile mask; larger ones are
// counted and written a tile row at a time.
constexpr uint32_t kWarpArea = 128;
constexpr uint32_t kMaskArea = kWarpArea;
static_assert(kMaskArea <= 128, "a tile mask has 128 bits");

// ---- Splats of more than kWarpArea tiles, one tile row at a time ----
//
// The tiles of a row that the exact test (tile_touched) accepts are those
// whose box of pixel centres meets the ellipse {power <= cutoff}; within the
// row's band of pixel centres, the ellipse spans one x interval [XL, XR]. In
// double precision that interval gives, with a margin m covering every
// rounding of the float test (its inputs' rounding and the power's, which
// grows with the conic's condition number), the columns that are certainly
// touched and the few around them that must be tested exactly. A row is then
// counted in O(1) plus a handful of exact tests, and its pairs are the
// certain run with the exact hits either side of it: the counts and pairs
// are the per-tile test's own, at a cost that follows the pairs, not the
// rectangle's area. Rows near the top or bottom of the ellipse, and
// ill-conditioned conics, are tested tile by tile.
struct Footprint {
    float cx, cy, a, b, c, cut;
    uint32_t x0, x1;      // the rectangle's columns
    uint32_t y0;          // its first row
    uint32_t tid;         // the splat's thread in the block
    uint32_t table;       // the splat's first row in the row table, or kNoTable
};
constexpr uint32_t kNoTable = 0xFFFFFFFFu;

struct RowPlan {
    int32_t lo, hi;           // candidate columns, inside the rectangle (none when lo > hi)
    int32_t sureLo, sureHi;   // certainly touched columns, inside [lo, hi] (none when sureLo > sureHi)
};

// The x range of tile column t's pixel centres, relative to the centre, as
// tile_touched forms it (the same float values, here exact in double).
__device__ __forceinline__ double col_lo(int32_t t, float cx) {
    return static_cast<double>(static_cast<float>(t * static_cast<int32_t>(kTile)) + 0.5f) - static_cast<double>(cx);
}
__device__ __forceinline__ double col_hi(int32_t t, uint32_t width, float cx) {
    const int32_t last = min((t + 1) * static_cast<int32_t>(kTile), static_cast<int32_t>(width)) - 1;
    return static_cast<double>(static_cast<float>(last) + 0.5f) - static_cast<double>(cx);
}

__device__ __forceinline__ RowPlan row_plan(const Footprint& fp, uint32_t ty, uint32_t width, uint32_t height) {
    RowPlan p{static_cast<int32_t>(fp.x0), static_cast<int32_t>(fp.x1), 1, 0};   // default: every column exact
    const double a = fp.a, b = fp.b, c = fp.c, k = fp.cut;
    const double det = a * c - b * b;
    if (!(a > 0.0) || !(c > 0.0) || !(k > 0.0) || !(det > 1e-6 * a * c)) return p;
    const double hx = sqrt(k * c / det), hy = sqrt(k * a / det);
    // Margin: the float test's power carries a relative error of a few
    // roundings (4 x 2^-24) times the condition number kappa, which moves
    // the boundary by at most that times half the long axis; its box
    // coordinates carry one rounding of magnitudes up to |centre| + extent.
    // Both with a factor of 8 to spare, plus a quarter pixel.
    const double lmin = 0.5 * (a + c) - sqrt(0.25 * (a - c) * (a - c) + b * b);
    if (!(lmin > 0.0)) return p;
    const double kappa = (fabs(a) + 2.0 * fabs(b) + fabs(c)) / lmin;
    const double reach = fabs(static_cast<double>(fp.cx)) + fabs(static_cast<double>(fp.cy)) + hx + hy + 64.0;
    const double m = 0.25 + 1.0e-6 * kappa * (hx + hy) + 5.0e-7 * reach;
    if (!(m < 24.0)) return p;
    const int32_t ity = static_cast<int32_t>(ty);
    const double ylo = static_cast<double>(static_cast<float>(ity * static_cast<int32_t>(kTile)) + 0.5f) -
                       static_cast<double>(fp.cy);
    const int32_t lastRow = min((ity + 1) * static_cast<int32_t>(kTile), static_cast<int32_t>(height)) - 1;
    const double yhi = static_cast<double>(static_cast<float>(lastRow) + 0.5f) - static_cast<double>(fp.cy);
    if (yhi < -hy - m || ylo > hy + m) {   // the band misses the ellipse by more than the margin
        p.lo = 1;
        p.hi = 0;
        return p;
    }
    // Near the ellipse's top or bottom the band's x extent is ill-conditioned
    // (it grows as the square root of the band's overlap): there the
    // candidates are the x extent of the band widened by m on both sides,
    // each tested exactly, and none is certain.
    const bool tangent = yhi < -hy + m || ylo > hy - m;
    const double bandLo = tangent ? fmax(ylo - m, -hy) : ylo;
    const double bandHi = tangent ? fmin(yhi + m, hy) : yhi;
    // The ellipse's x extent within the band: its leftmost and rightmost
    // points (x = -+hx, y = -b x / c) clamped into the band.
    const double yl = fmin(fmax(b * hx / c, bandLo), bandHi);
    const double yr = fmin(fmax(-b * hx / c, bandLo), bandHi);
    const double xl = (-b * yl - sqrt(fmax(k * a - det * yl * yl, 0.0))) / a;
    const double xr = (-b * yr + sqrt(fmax(k * a - det * yr * yr, 0.0))) / a;
    // First column whose hi >= v, and last whose lo <= v, within the
    // rectangle (the estimate is exact but for the clipped last column; the
    // adjustment steps are bounded and, if they do not settle, every column
    // is tested exactly).
    const int32_t x0 = static_cast<int32_t>(fp.x0), x1 = static_cast<int32_t>(fp.x1);
    bool ok = true;
    auto firstHiAtLeast = [&](double v) -> int32_t {
        const double e = ceil((v + static_cast<double>(fp.cx) - 15.5) / 16.0);
        int32_t t = static_cast<int32_t>(fmin(fmax(e, static_cast<double>(x0)), static_cast<double>(x1 + 1)));
        for (int it = 0; it < 3 && t > x0 && col_hi(t - 1, width, fp.cx) >= v; ++it) --t;
        for (int it = 0; it < 3 && t <= x1 && col_hi(t, width, fp.cx) < v; ++it) ++t;
        if ((t > x0 && col_hi(t - 1, width, fp.cx) >= v) || (t <= x1 && col_hi(t, width, fp.cx) < v)) ok = false;
        return t;
    };
    auto lastLoAtMost = [&](double v) -> int32_t {
        const double e = floor((v + static_cast<double>(fp.cx) - 0.5) / 16.0);
        int32_t t = static_cast<int32_t>(fmin(fmax(e, static_cast<double>(x0 - 1)), static_cast<double>(x1)));
        for (int it = 0; it < 3 && t < x1 && col_lo(t + 1, fp.cx) <= v; ++it) ++t;
        for (int it = 0; it < 3 && t >= x0 && col_lo(t, fp.cx) > v; ++it) --t;
        if ((t < x1 && col_lo(t + 1, fp.cx) <= v) || (t >= x0 && col_lo(t, fp.cx) > v)) ok = false;
        return t;
    };
    const int32_t lo = firstHiAtLeast(xl - m), hi = lastLoAtMost(xr + m);
    const int32_t sureLo = tangent ? 1 : firstHiAtLeast(xl + m), sureHi = tangent ? 0 : lastLoAtMost(xr - m);
    if (!ok) return p;
    p.lo = lo;
    p.hi = hi;
    p.sureLo = tangent ? 1 : max(sureLo, lo);
    p.sureHi = tangent ? 0 : min(sureHi, hi);
    return p;
}

// A row's touched tiles in column order: `visit(t)` for each exact hit and
// `run(t0, t1)` for the certain run [t0, t1].
template <class Hit, class Run>
__device__ __forceinline__ void row_walk(const Footprint& fp, uint32_t ty, uint32_t width, uint32_t height,
                                         Hit&& visit, Run&& run) {
    const RowPlan p = row_plan(fp, ty, width, height);
    const bool sure = p.sureLo <= p.sureHi;
    const int32_t leftEnd = sure ? p.sureLo - 1 : p.hi;
    for (int32_t t = p.lo; t <= leftEnd; ++t)
        if (tile_touched(width, height, fp.cx, fp.cy, fp.a, fp.b, fp.c, fp.cut, static_cast<uint32_t>(t), ty)) visit(t);
    if (!sure) return;
    run(p.sureLo, p.sureHi);
    for (int32_t t = p.sureHi + 1; t <= p.hi; ++t)
        if (tile_touched(width, height, fp.cx, fp.cy, fp.a, fp.b, fp.c, fp.cut, static_cast<uint32_t>(t), ty)) visit(t);
}

// One row: its count, first and last touched column, and whether its hits
// are one run.
struct RowCount {
    uint32_t count;
    int32_t first, last;
    bool regular;
};
__device__ __forceinline__ RowCount row_count(const Footprint& fp, uint32_t r, uint32_t width, uint32_t height) {
    RowCount rc{0, 0, -2, true};
    auto add = [&](int32_t t0, int32_t t1) {
        if (rc.count != 0 && t0 != rc.last + 1) rc.regular = false;
        if (rc.count == 0) rc.first = t0;
        rc.count += static_cast<uint32_t>(t1 - t0 + 1);
        rc.last = t1;
    };
    row_walk(fp, fp.y0 + r, width, height, [&](int32_t t) { add(t, t); }, add);
    return rc;
}
constexpr uint64_t kFlagAggregate = 1ull << 62;
constexpr uint64_t kFlagInclusive = 2ull << 62;
constexpr uint64_t kValueMask = (1ull << 62) - 1;
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* sWarp, uint32_t* total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, x, d);
        if (lane >= d) x += o;
    }
    if (lane == 31) sWarp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kProjectThreads / 32 ? sWarp[lane] : 0;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, w, d);
            if (lane >= d) w += o;
        }
        if (lane < kProjectThreads / 32) sWarp[lane] = w;
    }
    __syncthreads();
    const uint32_t before = warp == 0 ? 0 : sWarp[warp - 1];
    *total = sWarp[kProjectThreads / 32 - 1];
    __syncthreads();
    return before + x - v;
}

// The block's first pair in the frame: warp 0 publishes the block's total
// and looks back 32 partitions at a time (lane l reads the status of
// partition q - l); the nearest inclusive prefix ends the walk and the
// aggregates up to it are summed across the warp. A partition in the window
// that has published nothing yet makes the warp read the window again
// (bounded: after kSpinLimit polls kErrTimeout is raised and the walk
// ends). The frame's last partition writes the pair total to counters[1].
// Called by warp 0 only; lane 0's result is the block's base.
__device__ __forceinline__ unsigned long long frame_lookback(uint64_t* __restrict__ status, uint32_t g,
                                                             uint32_t lastPartition, uint32_t blockTotal,
                                                             uint32_t* __restrict__ counters,
                                                             uint32_t* __restrict__ err) {
    const uint32_t lane = threadIdx.x & 31u;
    uint64_t prefix = 0;
    if (lane == 0) {
        cuda::atomic_ref<uint64_t, cuda::thread_scope_device> mine(status[g]);
        mine.store((g == 0 ? kFlagInclusive : kFlagAggregate) | blockTotal, cuda::memory_order_relaxed);
    }
    if (g > 0) {
        int64_t q = static_cast<int64_t>(g) - 1;
        uint32_t spins = 0;
        while (true) {
            const int64_t idx = q - static_cast<int64_t>(lane);
            uint64_t word = kFlagInclusive;   // before partition 0: an empty inclusive prefix
            if (idx >= 0) {
                cuda::atomic_ref<uint64_t, cuda::thread_scope_device> sref(status[idx]);
                word = sref.load(cuda::memory_order_relaxed);
            }
            const uint32_t inclusive = __ballot_sync(0xFFFFFFFFu, (word & kFlagInclusive) != 0);
            const uint32_t empty = __ballot_sync(0xFFFFFFFFu, (word & ~kValueMask) == 0);
            const uint32_t first = inclusive != 0 ? static_cast<uint32_t>(__ffs(inclusive)) - 1u : 32u;
            const uint32_t upTo = first < 32u ? (2u << first) - 1u : 0xFFFFFFFFu;   // lanes 0..first
            if ((empty & upTo) != 0) {
                if (++spins > kSpinLimit) {
                    if (lane == 0) atomicOr(err, kErrTimeout);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            uint64_t v = ((upTo >> lane) & 1u) ? (word & kValueMask) : 0ull;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
            prefix += v;
            if (first < 32u) break;
            q -= 32;
        }
        if (lane == 0) {
            cuda::atomic_ref<uint64_t, cuda::thread_scope_device> mine(status[g]);
            mine.store(kFlagInclusive | (prefix + blockTotal), cuda::memory_order_relaxed);
        }
    }
    if (lane == 0 && g == lastPartition) {
        const uint64_t all = prefix + blockTotal;
        if (all > 0xFFFFFFFFull) atomicOr(err, kErrTooManyPairs);
        counters[1] = static_cast<uint32_t>(all);
    }
    return prefix;
}

// The position of the r-th set bit (from 0, lowest first) of a 64-bit mask
// that has more than r set bits: the half, then five halvings by population
// count.
__device__ __forceinline__ uint32_t nth_set_bit(unsigned long long m, uint32_t r) {
    uint32_t w = static_cast<uint32_t>(m);
    uint32_t base = 0;
    const uint32_t lowCount = static_cast<uint32_t>(__popc(w));
    if (r >= lowCount) {
        r -= lowCount;
        w = static_cast<uint32_t>(m >> 32);
        base = 32;
    }
#pragma unroll
    for (uint32_t width = 16; width > 0; width >>= 1) {
        const uint32_t lowBits = w & ((1u << width) - 1u);
        const uint32_t c = static_cast<uint32_t>(__popc(lowBits));
        if (r >= c) {
            r -= c;
            w >>= width;
            base += width;
        } else {
            w = lowBits;
        }
    }
    return base;
}

// The same over a 128-bit mask (lo, hi) with more than r set bits.
__device__ __forceinline__ uint32_t nth_set_bit128(unsigned long long lo, unsigned long long hi, uint32_t r) {
    const uint32_t lowCount = static_cast<uint32_t>(__popcll(lo));
    return r < lowCount ? nth_set_bit(lo, r) : 64u + nth_set_bit(hi, r - lowCount);
}

// Row and column of bit `bit` of a row-major mask of width w (w <= 128,
// bit < 128): (bit + 1/2) / w in float lies at least 1/256 away from an
// integer, far more than its rounding error, so the floor is exact.
__device__ __forceinline__ void mask_bit_tile(uint32_t bit, uint32_t w, float invW, uint32_t& dx, uint32_t& dy) {
    dy = static_cast<uint32_t>((static_cast<float>(bit) + 0.5f) * invW);
    dx = bit - dy * w;
}

struct PairSink {
    unsigned long long* pairs;
    uint32_t* values;     // training, emit index as a sort value
    uint32_t* emitSlot;   // training, emit index as the low field
    uint32_t capacity;
    uint32_t* err;
    // `word` holds the tile and the depth key above the low field, which is
    // filled here: the slot, or the emit index itself.
    __device__ __forceinline__ void put(uint64_t at, unsigned long long word, uint32_t slot) const {
        if (at < capacity) {
            if (emitSlot != nullptr) {
                pairs[at] = word | at;
                emitSlot[at] = slot;
            } else {
                pairs[at] = word | slot;
                if (values != nullptr) values[at] = static_cast<uint32_t>(at);
            }
        } else {
            atomicOr(err, kErrOverflow);
        }
    }
};

// A PairSink that also counts, in shared memory, the tile sort's digits of
// every pair it writes (the tile's low byte, and its second byte when the
// sort takes two passes), so that the sort needs no counting pass of its own.
struct CountingSink {
    PairSink inner;
    uint32_t* digits;   // shared: 256 a pass
    uint32_t passes;    // 1 or 2
    __device__ __forceinline__ void put(uint64_t at, unsigned long long word, uint32_t slot) const {
        if (at < inner.capacity) {
            const uint32_t tile = static_cast<uint32_t>(word >> 32);
            atomicAdd(&digits[tile & 0xFFu], 1u);
            if (passes > 1) atomicAdd(&digits[256 + ((tile >> 8) & 0xFFu)], 1u);
        }
        inner.put(at, word, slot);
    }
};

// The block's large splats counted a tile row per thread per step (rows in
// list order, splat after splat): counts added into counts[splat thread]
// (bit 31 marks a splat with a row that is not one run); each row's first
// column and count also kept in the row table for a splat that has a place
// there, so that writing its pairs needs no second row plan.
__device__ __forceinline__ void count_large_rows(const Footprint* foot, const uint32_t* footRow, uint32_t bigTotal,
                                                 uint32_t rowsTotal, uint32_t width, uint32_t height, uint32_t* counts,
                                                 uint2* __restrict__ rowTable) {
    const uint32_t tid = threadIdx.x;
    uint32_t fs = 0;   // the splat of row item j: found by search once, then advanced
    {
        uint32_t lo = 0, hi = bigTotal;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (footRow[mid] <= tid) lo = mid; else hi = mid;
        }
        fs = lo;
    }
    for (uint32_t j = tid; j < rowsTotal; j += kProjectThreads) {
        while (footRow[fs + 1] <= j) ++fs;
        const Footprint fp = foot[fs];
        const uint32_t r = j - footRow[fs];
        const RowCount rc = row_count(fp, r, width, height);
        if (rc.count != 0) atomicAdd(&counts[fp.tid], rc.count);
        if (!rc.regular) atomicOr(&counts[fp.tid], 0x80000000u);
        if (fp.table != kNoTable) rowTable[fp.table + r] = make_uint2(static_cast<uint32_t>(rc.first), rc.count);
    }
}

// The pairs of the block's large, unmasked splats whose rows are single runs:
// a chunk of 256 rows at a time, each row's count and first column from its
// row plan (as when counting) and its pairs' place among the chunk's by a
// block scan; then each warp writes whole rows, its lanes on consecutive
// pairs of a row. takenStart[t]: the pairs of such splats before splat t.
// slotOf[t]: the slot of the block's splat t (null: slotBase + t).
template <class Sink>
__device__ __forceinline__ void emit_large_rows(const Footprint* foot, const uint32_t* footRow, uint32_t bigTotal,
                                             uint32_t rowsTotal, uint32_t width, uint32_t height, uint32_t tileBase,
                                             uint32_t tilesX, const uint32_t* widthBits, const uint32_t* start,
                                             const uint32_t* takenStart, const unsigned long long* low,
                                             uint32_t* scanScratch, unsigned long long blockBase, uint32_t tileShift,
                                             uint32_t slotBase, const uint32_t* slotOf, const Sink& sink,
                                             const uint2* __restrict__ rowTable = nullptr) {
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    uint32_t fs = 0;
    {
        uint32_t lo = 0, hi = bigTotal;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (footRow[mid] <= tid) lo = mid; else hi = mid;
        }
        fs = lo;
    }
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < rowsTotal; c0 += kProjectThreads) {
        const uint32_t j = c0 + tid;
        uint32_t cnt = 0, first = 0, meta = 0;
        if (j < rowsTotal) {
            while (footRow[fs + 1] <= j) ++fs;
            const Footprint fp = foot[fs];
            if ((widthBits[fp.tid] & 0x80000000u) == 0) {
                const uint32_t r = j - footRow[fs];
                if (fp.table != kNoTable) {   // kept by the projection's count
                    const uint2 e = rowTable[fp.table + r];
                    cnt = e.y;
                    first = e.x;
                } else {
                    const RowCount rc = row_count(fp, r, width, height);
                    cnt = rc.count;
                    first = static_cast<uint32_t>(rc.first);
                }
                meta = (fp.y0 + r) | (fp.tid << 16);
            }
        }
        uint32_t chunkTotal = 0;
        const uint32_t off = block_exclusive_scan(cnt, scanScratch, &chunkTotal);
        // Each warp writes the pairs of its 32 rows (a lane's own row) 32 at a
        // time, lanes on consecutive pairs: a lane finds its pair's row by a
        // binary search over the warp's running counts (shuffles: the last
        // lane whose count starts at or before the pair, which always has
        // pairs), so short rows leave no lane idle.
        unsigned long long at0 = 0, word0 = 0;
        uint32_t slot = 0;
        if (cnt != 0) {
            const uint32_t ty = meta & 0xFFFFu, owner = meta >> 16;
            at0 = blockBase + start[owner] + (carry + off - takenStart[owner]);
            word0 = (static_cast<unsigned long long>(tileBase + ty * tilesX + first) << tileShift) | low[owner];
            slot = slotOf != nullptr ? slotOf[owner] : slotBase + owner;
        }
        uint32_t incl = cnt;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= d) incl += o;
        }
        const uint32_t warpTotal = __shfl_sync(0xFFFFFFFFu, incl, 31);
        const uint32_t excl = incl - cnt;
        for (uint32_t p0 = 0; p0 < warpTotal; p0 += 32) {
            const uint32_t pos = p0 + lane;
            uint32_t l = 0;
#pragma unroll
            for (uint32_t step = 16; step >= 1; step >>= 1) {
                const uint32_t e = __shfl_sync(0xFFFFFFFFu, excl, static_cast<int>(l + step));
                if (e <= pos) l += step;
            }
            const int src = static_cast<int>(l);
            const uint32_t k = pos - __shfl_sync(0xFFFFFFFFu, excl, src);
            const unsigned long long at = __shfl_sync(0xFFFFFFFFu, at0, src);
            const unsigned long long word = __shfl_sync(0xFFFFFFFFu, word0, src);
            const uint32_t slotHere = __shfl_sync(0xFFFFFFFFu, slot, src);
            if (pos < warpTotal) sink.put(at + k, word + (static_cast<unsigned long long>(k) << tileShift), slotHere);
        }
        carry += chunkTotal;
        __syncthreads();
    }
}

// The pairs of a warp's splats whose tiles are tested one by one (large
// splats with a row that is not one run, possible only through the float
// test's rounding at the ellipse's edge): for each such splat the warp
// repeats the exact tile test
// over its rectangle, 32 tiles at a time, and writes the hits in row-major
// order. The splat's record is read back from `records` (written earlier by
// its thread): records[slotOf ? slotOf[s] : s].
template <class Sink>
__device__ __forceinline__ void emit_by_warp(bool mine, uint32_t area, const uint32_t* widthBits,
                                          const uint32_t* rectBits, const uint32_t* start,
                                          const unsigned long long* low, const ProjRecord* records, uint32_t width,
                                          uint32_t height, uint32_t tileBase, uint32_t tilesX,
                                          unsigned long long blockBase, uint32_t tileShift, uint32_t slotBase,
                                          const uint32_t* slotOf, const Sink& sink) {
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    uint32_t todo = __ballot_sync(0xFFFFFFFFu, mine);
    while (todo != 0) {
        const int src = __ffs(todo) - 1;
        todo &= todo - 1;
        const uint32_t s = (tid & ~31u) + static_cast<uint32_t>(src);
        const uint32_t sArea = __shfl_sync(0xFFFFFFFFu, area, src);
        const ProjRecord rec = records[slotOf != nullptr ? slotOf[s] : s];
        const uint32_t sW = widthBits[s] & 0xFFFFu;
        const uint32_t sX = rectBits[s] & 0xFFFFu, sY = rectBits[s] >> 16;
        unsigned long long at = blockBase + start[s];
        const unsigned long long lowWord = low[s];
        const uint32_t stepDy = 32u / sW, stepDx = 32u % sW;
        uint32_t dx = lane % sW, dy = lane / sW;
        for (uint32_t base = 0; base < sArea; base += 32) {
            const uint32_t tx = sX + dx, ty = sY + dy;
            const bool hit = base + lane < sArea &&
                             tile_touched(width, height, rec.screen.x, rec.screen.y, rec.conic.x, rec.conic.y,
                                          rec.conic.z, rec.screen.w, tx, ty);
            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, hit);
            if (hit) {
                sink.put(at + static_cast<uint32_t>(__popc(bal & ((1u << lane) - 1u))),
                         (static_cast<unsigned long long>(tileBase + ty * tilesX + tx) << tileShift) | lowWord,
                         slotOf != nullptr ? slotOf[s] : slotBase + s);
            }
            at += static_cast<uint32_t>(__popc(bal));
            dx += stepDx;
            dy += stepDy;
            if (dx >= sW) {
                dx -= sW;
                dy += 1;
            }
        }
    }
}


// kEmit: emit the pairs (offsets by look-back over the frame's partitions).
// Otherwise stop after the records and counts, and write per slot the
// depth word (depth key << 32 | slot) the depth sort orders and the two aux
// words emit_pairs_kernel reads: the tile mask of a masked splat, else 1 when
// a row of a large splat's hits is not one run.
template <class Src, bool kEmit = true, bool kChained = false>
__global__ void __launch_bounds__(kProjectThreads, 4)
project_emit_kernel(FrameParams fArg, const FrameParams* __restrict__ fDev, Src src, TrainOutputs train,
                    uint32_t stageWords, uint32_t shVector,
                    ProjRecord* __restrict__ proj, uint4* __restrict__ rects, uint32_t* __restrict__ touchedOut,
                    uint32_t* __restrict__ keysOut, uint32_t* __restrict__ counters, uint64_t* __restrict__ status,
                    uint32_t* __restrict__ ticket, uint32_t partitionBase, uint32_t lastPartition, uint32_t lowBits,
                    unsigned long long* __restrict__ pairs, uint32_t capacity,
                    unsigned long long* __restrict__ auxOut = nullptr,
                    unsigned long long* __restrict__ depthWordsOut = nullptr,
                    uint32_t* __restrict__ depthDigits = nullptr, uint2* __restrict__ rowTable = nullptr,
                    uint32_t rowCap = 0) {
    chained_entry<kChained>();
    extern __shared__ __align__(16) uint32_t shStage[];
    __shared__ uint32_t sPart;
    __shared__ uint32_t sScan[kProjectThreads / 32];
    __shared__ uint32_t sStart[kProjectThreads + 1];       // block-relative pair offset of each splat
    __shared__ uint32_t sSmallStart[kProjectThreads + 1];  // the same over masked splats only
    __shared__ unsigned long long sLow[kProjectThreads];   // depth key << lowBits
    __shared__ uint32_t sRect[kProjectThreads];            // x0 | y0 << 16
    __shared__ uint32_t sWidth[kProjectThreads];
    __shared__ Footprint sFoot[kProjectThreads];           // the block's splats of more than kWarpArea tiles
    __shared__ uint32_t sFootRow[kProjectThreads + 1];     // their first row in the block's row list
    __shared__ unsigned long long sBase;
    // The frame's parameters: by value, or (when a captured graph replays a
    // batch with new cameras) read from device memory, once per block.
    __shared__ FrameParams sF;
    // Without emission: the block's counts of the depth keys' three bytes
    // (the depth sort's digits), added to depthDigits at the end.
    __shared__ uint32_t sDigits[kEmit ? 1 : 3 * 256];
    uint32_t* err = counters + 2;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    if (tid == 0) {
        sPart = atomicAdd(ticket, 1u);
        sF = fDev != nullptr ? *fDev : fArg;
    }
    if constexpr (!kEmit) {
        for (uint32_t k = tid; k < 3 * 256; k += kProjectThreads) sDigits[k] = 0;
    }
    __syncthreads();
    const FrameParams& f = sF;
    const uint32_t part = sPart;
    const uint32_t blockStart = part * kProjectThreads;
    const uint32_t i = blockStart + tid;
    const bool inRange = i < f.count;

    // Harmonics of the whole block, in flight while the geometry runs.
    if (stageWords != 0 && blockStart < f.count) {
        const uint32_t nBlock = min(kProjectThreads, f.count - blockStart);
        const uint32_t words = nBlock * f.shWords;
        const uint32_t* rows = src.sh + static_cast<size_t>(blockStart) * f.shWords;
        uint32_t w0 = 0;
        if (shVector) {
            const uint32_t nvec = words >> 2;
            for (uint32_t v = tid; v < nvec; v += kProjectThreads) cp_async16(&shStage[v * 4], rows + v * 4);
            w0 = nvec * 4;
        }
        for (uint32_t w = w0 + tid; w < words; w += kProjectThreads) cp_async4(&shStage[w], rows + w);
    }

    bool alive = false;
    float3 p = make_float3(0.0f, 0.0f, 0.0f);
    float3 t = p;
    float cx = 0.0f, cy = 0.0f, ca = 0.0f, cb = 0.0f, cc = 0.0f, alpha = 0.0f, cutoff = 0.0f;
    uint4 rect = make_uint4(1, 1, 0, 0);
    Fate fate{true, false, 0.0f};
    typename Src::Loaded loaded{};
    if constexpr (Src::kDisc) {
        // points_project.slang:40-70: a disc of the point's radius, cut at
        // one radius (conic 1/r^2 on the diagonal), alpha one.
        if (inRange) {
            const float4 po = __ldg(src.positions + i);
            p = make_float3(po.x, po.y, po.z);
            t = to_view(f, p);
            alive = (t.z > f.nearZ) && !(t.z > f.farZ);
            if (alive) {
                const float radius = src.radius(f, t.z);
                const float invZ = f.ortho != 0 ? 1.0f : 1.0f / t.z;
                cx = f.focalX * t.x * invZ + f.centreX;
                cy = f.focalY * t.y * invZ + f.centreY;
                ca = 1.0f / (radius * radius);
                cb = 0.0f;
                cc = 1.0f / (radius * radius);
                alpha = 1.0f;
                cutoff = 1.0f;
                // tileRect, frame.slang:149-161, with the radius as the extent
                const float x1 = cx - radius, y1 = cy - radius, x2 = cx + radius, y2 = cy + radius;
                if (x2 < 0.0f || y2 < 0.0f || x1 >= static_cast<float>(f.width) ||
                    y1 >= static_cast<float>(f.height)) {
                    alive = false;
                } else {
                    rect = make_uint4(static_cast<uint32_t>(fmaxf(x1, 0.0f)) / kTile,
                                      static_cast<uint32_t>(fmaxf(y1, 0.0f)) / kTile,
                                      static_cast<uint32_t>(fminf(x2, static_cast<float>(f.width) - 1.0f)) / kTile,
                                      static_cast<uint32_t>(fminf(y2, static_cast<float>(f.height) - 1.0f)) / kTile);
                    alive = !(rect.x > rect.z || rect.y > rect.w);
                }
            }
        }
    } else if (inRange) {
        float opacity;
        float3 scale;
        src.load(i, loaded, p, opacity, scale);
        fate = edit_fate(f.edit, p, opacity, scale);
        t = to_view(f, p);
        alive = !fate.removed && (t.z > f.nearZ) && !(t.z > f.farZ);
        if (alive) {
            float x, y, z, w;
            src.rotation(loaded, x, y, z, w);
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
                const float tx = clampf(t.x * invZ, limLoX, limHiX) * t.z;
                const float ty = clampf(t.y * invZ, limLoY, limHiY) * t.z;
                jx0 = f.focalX * invZ; jx1 = 0.0f; jx2 = -f.focalX * tx * invZ * invZ;
                jy0 = 0.0f; jy1 = f.focalY * invZ; jy2 = -f.focalY * ty * invZ * invZ;
            }
            // mul(row, W), then mul(row, M): result[j] = row0 X[0][j] + row1 X[1][j] + row2 X[2][j]
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
                alpha = fate.opacity;
                if (f.antialias != 0) alpha = alpha * sqrtf(fmaxf(detBefore, 0.0f) / det);
                alive = alpha >= 1.0f / 255.0f;
            }
            if (alive) {
                ca = c / det;
                cb = -b / det;
                cc = a / det;
                cutoff = cutoff_power(alpha);
                // footprintExtent, frame.slang:142-146
                const float det2 = ca * cc - cb * cb;
                const float inv = det2 > 1e-20f ? 1.0f / det2 : 0.0f;
                const float ex = sqrtf(fmaxf(cutoff * cc * inv, 0.0f));
                const float ey = sqrtf(fmaxf(cutoff * ca * inv, 0.0f));
                // tileRect, frame.slang:149-161
                const float x1 = cx - ex, y1 = cy - ey, x2 = cx + ex, y2 = cy + ey;
                if (x2 < 0.0f || y2 < 0.0f || x1 >= static_cast<float>(f.width) ||
                    y1 >= static_cast<float>(f.height)) {
                    alive = false;
                } else {
                    rect = make_uint4(static_cast<uint32_t>(fmaxf(x1, 0.0f)) / kTile,
                                      static_cast<uint32_t>(fmaxf(y1, 0.0f)) / kTile,
                                      static_cast<uint32_t>(fminf(x2, static_cast<float>(f.width) - 1.0f)) / kTile,
                                      static_cast<uint32_t>(fminf(y2, static_cast<float>(f.height) - 1.0f)) / kTile);
                    alive = !(rect.x > rect.z || rect.y > rect.w);
                }
            }
        }
    }

    // The exact touched count (splat_project.slang:148-160), row-major over
    // the rectangle. Up to kMaskArea tiles a bitmask of the touched tiles is
    // kept, bit k for the rectangle's k-th tile in row-major order (two
    // words); such splats are "masked" and their pairs are written from it.
    const uint32_t rw = alive ? rect.z - rect.x + 1 : 0;
    const uint32_t rh = alive ? rect.w - rect.y + 1 : 0;
    const uint32_t area = rw * rh;
    const uint32_t sh = rw <= 1 ? 0u : 32u - static_cast<uint32_t>(__clz(rw - 1));
    const bool masked = alive && area <= kMaskArea;
    uint32_t touched = 0;
    unsigned long long mask = 0, maskHi = 0;
    // Splats of up to kWarpArea tiles: the warp tests their tiles together,
    // 32 (splat, tile) pairs a step in lane and row-major tile order, so that
    // no lane waits on a neighbour with more tiles and no step is left part
    // empty at the end of a splat. A lane finds its pair's splat by a binary
    // search over the warp's running tile counts (shuffles: the last lane
    // whose count starts at or before the pair, which always has tiles), and
    // each splat's lane takes its run of the step's ballot as mask bits.
    {
        const uint32_t mine = alive && area <= kWarpArea ? area : 0u;
        uint32_t incl = mine;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= d) incl += o;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        const uint32_t excl = incl - mine;
        const float invW = mine != 0 ? 1.0f / static_cast<float>(rw) : 0.0f;
        const float gate = mine != 0 ? far_edge_gate(ca, cb, cc, cutoff) : INFINITY;
        for (uint32_t c0 = 0; c0 < total; c0 += 32) {
            const uint32_t pos = c0 + lane;
            uint32_t l = 0;
#pragma unroll
            for (uint32_t step = 16; step >= 1; step >>= 1) {
                const uint32_t e = __shfl_sync(0xFFFFFFFFu, excl, static_cast<int>(l + step));
                if (e <= pos) l += step;
            }
            const int src = static_cast<int>(l);
            const uint32_t k = pos - __shfl_sync(0xFFFFFFFFu, excl, src);
            const uint32_t oW = __shfl_sync(0xFFFFFFFFu, rw, src);
            const float oInv = __shfl_sync(0xFFFFFFFFu, invW, src);
            const uint32_t oX = __shfl_sync(0xFFFFFFFFu, rect.x, src), oY = __shfl_sync(0xFFFFFFFFu, rect.y, src);
            const float ocx = __shfl_sync(0xFFFFFFFFu, cx, src), ocy = __shfl_sync(0xFFFFFFFFu, cy, src);
            const float oa = __shfl_sync(0xFFFFFFFFu, ca, src), ob = __shfl_sync(0xFFFFFFFFu, cb, src);
            const float oc = __shfl_sync(0xFFFFFFFFu, cc, src), ocut = __shfl_sync(0xFFFFFFFFu, cutoff, src);
            const float ogate = __shfl_sync(0xFFFFFFFFu, gate, src);
            uint32_t dx = 0, dy = 0;
            mask_bit_tile(k, oW, oInv, dx, dy);
            const bool hit = pos < total && tile_touched(f.width, f.height, ocx, ocy, oa, ob, oc, ocut, oX + dx, oY + dy,
                                                         ogate);
            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, hit);
            if (mine != 0) {
                const uint32_t lo = max(excl, c0), hi = min(incl, c0 + 32);
                if (lo < hi) {
                    const unsigned long long run = ((static_cast<unsigned long long>(bal) >> (lo - c0)) &
                                                    ((1ull << (hi - lo)) - 1ull));
                    const uint32_t at = lo - excl;   // the run's first bit in the 128-bit mask
                    if (at < 64) {
                        mask |= run << at;
                        if (at != 0) maskHi |= run >> (64 - at);   // bits past 63 (a run is at most 32 bits)
                    } else {
                        maskHi |= run << (at - 64);
                    }
                    touched += static_cast<uint32_t>(__popcll(run));
                }
            }
        }
    }
    // Larger splats are counted by the whole block below, a tile row at a
    // time, after the records are written (so that the projection's values
    // are no longer held in registers); the others are decided now.
    const bool bigHere = alive && area > kWarpArea;
    if (!bigHere) {
        alive = alive && touched != 0;
        if (!alive) touched = 0;
    }

    if (stageWords != 0) cp_async_wait_all();
    __syncthreads();

    const uint32_t slot = f.base + i;          // the slot in its view (pair words carry this)
    const uint32_t record = f.recordBase + slot;
    uint32_t key = 0x00FFFFFFu;
    if (inRange) {
        if (alive) {
            if constexpr (Src::kDisc) {
                ProjRecord rec;
                rec.screen = make_float4(cx, cy, t.z, cutoff);
                rec.conic = make_float4(ca, cb, cc, alpha);
                const float3 rgb = src.colour(i);   // colour.w one: an opaque disc
                rec.colour = make_float4(rgb.x, rgb.y, rgb.z, 1.0f);
                proj[record] = rec;
                if (f.writeDebug) rects[record] = rect;
                key = float_bits(t.z) >> 7;
            } else {
                const float3 base = src.base(loaded, shStage + tid * f.shWords);
                const uint32_t rpc = f.restPerColour;
                const uint32_t stored = rpc >= 15 ? 3u : rpc >= 8 ? 2u : rpc >= 3 ? 1u : 0u;
                const uint32_t degree = min(stored, f.shLimit);
                float3 restc = make_float3(0.0f, 0.0f, 0.0f);
                if (degree > 0) {
                    const float dx = p.x - f.eye[0], dy = p.y - f.eye[1], dz = p.z - f.eye[2];
                    const float l = sqrtf(dx * dx + dy * dy + dz * dz);
                    const float3 dir = make_float3(dx / l, dy / l, dz / l);
                    restc = evaluate_rest<Src::kRestOffset>(shStage + tid * f.shWords, degree, dir);
                }
                float3 colour = make_float3(fmaxf(base.x + restc.x, 0.0f), fmaxf(base.y + restc.y, 0.0f),
                                            fmaxf(base.z + restc.z, 0.0f));
                if (fate.graded) colour = edit_grade(f.edit, colour);
                ProjRecord rec;
                rec.screen = make_float4(cx, cy, t.z, cutoff);
                rec.conic = make_float4(ca, cb, cc, alpha);
                rec.colour = make_float4(colour.x, colour.y, colour.z, 0.0f);
                proj[record] = rec;
                if (f.writeDebug) rects[record] = rect;
                key = float_bits(t.z) >> 7;
            }
        } else {
            // splat_project.slang:39-49, plus a zeroed record
            ProjRecord rec;
            rec.screen = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            rec.conic = rec.screen;
            rec.colour = rec.screen;
            proj[record] = rec;
            if (f.writeDebug) rects[record] = make_uint4(1, 1, 0, 0);
        }
    }

    // The block counts its large splats a tile row per thread per step, into
    // sSmallStart (zeroed here; the block scan writes it later). A row whose
    // hits are not one run marks its splat (bit 31) for the per-tile
    // emission.
    uint32_t bigTotal = 0, rowsTotal = 0, bigIdx = 0;
    uint32_t rowTableAt = kNoTable;
    const bool anyBig = __syncthreads_or(bigHere ? 1 : 0) != 0;   // most blocks have none
    if (anyBig) {
        bigIdx = block_exclusive_scan(bigHere ? 1u : 0u, sScan, &bigTotal);
        const uint32_t rowStart = block_exclusive_scan(bigHere ? rh : 0u, sScan, &rowsTotal);
        sSmallStart[tid] = 0;
        if (bigHere) {
            // A place for the splat's rows in the row table (counters[3]
            // counts the rows asked for; a splat past the table's end keeps
            // none and its rows are planned again when its pairs are written).
            if (rowTable != nullptr) {
                const uint32_t at = atomicAdd(counters + 3, rh);
                if (at <= rowCap && rh <= rowCap - at) rowTableAt = at;
            }
            sFoot[bigIdx] = Footprint{cx, cy, ca, cb, cc, cutoff, rect.x, rect.z, rect.y, tid, rowTableAt};
            sFootRow[bigIdx] = rowStart;
        }
        if (tid == 0) sFootRow[bigTotal] = rowsTotal;
        __syncthreads();
    }
    if (rowsTotal != 0) {
        count_large_rows(sFoot, sFootRow, bigTotal, rowsTotal, f.width, f.height, sSmallStart, rowTable);
        __syncthreads();
    }
    bool irregular = false;
    if (bigHere) {
        const uint32_t v = sSmallStart[tid];
        touched = v & 0x7FFFFFFFu;
        irregular = (v & 0x80000000u) != 0;
        if (touched == 0) {   // no tile holds a pixel centre inside it: culled after all
            alive = false;
            key = 0x00FFFFFFu;
            ProjRecord rec;
            rec.screen = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            rec.conic = rec.screen;
            rec.colour = rec.screen;
            proj[record] = rec;
            if (f.writeDebug) rects[record] = make_uint4(1, 1, 0, 0);
        }
    }
    if (inRange) {
        if (f.writeDebug || train.offsets != nullptr) touchedOut[record] = touched;
        if (f.writeDebug) keysOut[record] = key;
    }
    const uint32_t ballot = __ballot_sync(0xFFFFFFFFu, inRange && alive);
    if (lane == 0 && ballot != 0) atomicAdd(counters, static_cast<uint32_t>(__popc(ballot)));
    if constexpr (!kEmit) {
        if (inRange) {
            reinterpret_cast<ulonglong2*>(auxOut)[record] =
                masked ? make_ulonglong2(mask, maskHi)
                       : make_ulonglong2((irregular ? 1ull : 0ull) | (static_cast<unsigned long long>(rowTableAt) << 32),
                                         0ull);
            depthWordsOut[record] = (static_cast<unsigned long long>(key) << 32) | slot;
            atomicAdd(&sDigits[key & 0xFFu], 1u);
            atomicAdd(&sDigits[256 + ((key >> 8) & 0xFFu)], 1u);
            atomicAdd(&sDigits[512 + (key >> 16)], 1u);
        }
        __syncthreads();
        for (uint32_t k = tid; k < 3 * 256; k += kProjectThreads) {
            const uint32_t v = sDigits[k];
            if (v != 0 && depthDigits != nullptr) atomicAdd(depthDigits + k, v);
        }
        return;
    }

    // Offsets: block scan, then decoupled look-back over the frame's partitions.
    uint32_t blockTotal = 0;
    const uint32_t start = block_exclusive_scan(touched, sScan, &blockTotal);
    sStart[tid] = start;
    const bool writeOffset = train.offsets != nullptr && inRange;
    sLow[tid] = static_cast<unsigned long long>(key) << lowBits;
    sRect[tid] = rect.x | (rect.y << 16);
    sWidth[tid] = rw | (sh << 16) | (irregular ? 0x80000000u : 0u);
    if (tid == 0) sStart[kProjectThreads] = blockTotal;
    if (tid < 32) sBase = frame_lookback(status, partitionBase + part, lastPartition, blockTotal, counters, err);
    __syncthreads();
    const unsigned long long blockBase = sBase;
    if (writeOffset) train.offsets[slot] = static_cast<uint32_t>(blockBase + start);
    const PairSink sink{pairs, train.values, train.emitSlot, capacity, err};
    const uint32_t tileShift = 24 + lowBits;
    const uint32_t slotBase = slot - tid;   // the slot of the block's first splat

    // Masked splats: each warp writes its own splats' pairs, 32 at a time,
    // consecutive lanes on consecutive pairs (a warp's splats' pairs follow
    // one another, so the writes are contiguous). A lane finds its pair's
    // splat by a binary search over the warp's running pair counts
    // (shuffles: the last lane whose count starts at or before the pair,
    // which always has pairs), and the tile as that splat's mask bit of the
    // same rank.
    {
        const uint32_t mine = masked ? touched : 0u;
        uint32_t incl = mine;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= d) incl += o;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        const uint32_t excl = incl - mine;
        const uint32_t mRect = rect.x | (rect.y << 16);
        const unsigned long long mLow = static_cast<unsigned long long>(key) << lowBits;
        const float mInvW = masked ? 1.0f / static_cast<float>(rw) : 0.0f;
        const uint32_t warpBase = slotBase + (tid & ~31u);
        for (uint32_t c0 = 0; c0 < total; c0 += 32) {
            const uint32_t pos = c0 + lane;
            uint32_t l = 0;
#pragma unroll
            for (uint32_t step = 16; step >= 1; step >>= 1) {
                const uint32_t e = __shfl_sync(0xFFFFFFFFu, excl, static_cast<int>(l + step));
                if (e <= pos) l += step;
            }
            const uint32_t r = pos - __shfl_sync(0xFFFFFFFFu, excl, static_cast<int>(l));
            const unsigned long long m = __shfl_sync(0xFFFFFFFFu, mask, static_cast<int>(l));
            const unsigned long long mH = __shfl_sync(0xFFFFFFFFu, maskHi, static_cast<int>(l));
            const uint32_t oRect = __shfl_sync(0xFFFFFFFFu, mRect, static_cast<int>(l));
            const uint32_t oW = __shfl_sync(0xFFFFFFFFu, rw, static_cast<int>(l));
            const float oInvW = __shfl_sync(0xFFFFFFFFu, mInvW, static_cast<int>(l));
            const uint32_t oStart = __shfl_sync(0xFFFFFFFFu, start, static_cast<int>(l));
            const unsigned long long oLow = __shfl_sync(0xFFFFFFFFu, mLow, static_cast<int>(l));
            if (pos < total) {
                uint32_t dx, dy;
                mask_bit_tile(nth_set_bit128(m, mH, r), oW, oInvW, dx, dy);
                const uint32_t tx = (oRect & 0xFFFFu) + dx;
                const uint32_t ty = (oRect >> 16) + dy;
                sink.put(blockBase + oStart + r,
                         (static_cast<unsigned long long>(f.tileBase + ty * f.tilesX + tx) << tileShift) | oLow,
                         warpBase + l);
            }
        }
    }
    // The rest (rectangles too large for a mask): the block writes their
    // pairs a chunk of 256 tile rows at a time, each row's count and first
    // column from its row plan (the same as when counting), flattened so
    // that consecutive threads write consecutive pairs. A splat's rows are in
    // order, so its pairs follow one another from its offset.
    if (rowsTotal != 0) {
        // Only the splats the rows walk (those in sFoot): their pairs' offsets
        // among the rows' pairs.
        const bool taken = touched != 0 && !masked && !irregular && area > kWarpArea;
        uint32_t takenTotal = 0;
        sSmallStart[tid] = block_exclusive_scan(taken ? touched : 0u, sScan, &takenTotal);
        __syncthreads();
        if (takenTotal != 0)
            emit_large_rows(sFoot, sFootRow, bigTotal, rowsTotal, f.width, f.height, f.tileBase, f.tilesX, sWidth,
                            sStart, sSmallStart, sLow, sScan, blockBase, tileShift,
                            slotBase, nullptr, sink);
    }
    // A splat whose rows are not all single runs (possible only through the
    // float test's rounding at the ellipse's edge): its warp repeats the exact
    // tile test over the rectangle, 32 tiles at a time.
    // Unmasked splats of up to kWarpArea tiles, and larger ones whose rows
    // are not all single runs: their warp writes their pairs, repeating the
    // exact tile test over the rectangle 32 tiles at a time.
    const bool byWarp = touched != 0 && !masked && (area <= kWarpArea || irregular);
    if (__ballot_sync(0xFFFFFFFFu, byWarp) != 0)
        emit_by_warp(byWarp, area, sWidth, sRect, sStart, sLow, proj + f.recordBase + slotBase, f.width, f.height,
                     f.tileBase, f.tilesX, blockBase, tileShift, slotBase, nullptr, sink);
}

// Stage (b) in depth order, as the reference emits (splat_emit.slang:17-50
// over the depth-sorted visible splats, TileRasterizer.cpp:418-438), in two
// kernels so that the pair writing keeps the projection's load balance:
//  - depth_offsets_kernel: each slot's first pair, the exclusive prefix of
//    the touched counts over the slots in depth order (block scan, then the
//    frame look-back; the last partition writes the total to counters[1]);
//  - emit_pairs_kernel: the pairs, written in slot order, each splat's at
//    its offset, as words tile << 32 | slot, its tiles in row-major order.
// Depth order puts the near splats, which are the large ones, together:
// writing their pairs in that order left a few blocks with most of a
// sort-heavy frame's pairs. In slot order they are spread over the grid as
// in the projection. A stable sort of the words on their tile bits then
// leaves every tile's pairs in (depth key, slot) order: the reference's
// two-sort order. Training frames keep the offsets (each slot's emit range
// is [offset, offset + touched)) and a way back from every pair to its emit
// index: the word's low field itself, with an emit index -> slot map
// (train.emitSlot), or a sort value beside a slot (train.values).
constexpr uint32_t kOffsetItems = 16;   // depth positions a thread

template <bool kChained>
__global__ void __launch_bounds__(kProjectThreads)
depth_offsets_kernel(const unsigned long long* __restrict__ sortedWords, uint32_t n,
                     const uint32_t* __restrict__ touchedIn, uint32_t* __restrict__ counters,
                     uint64_t* __restrict__ status, uint32_t* __restrict__ ticket, uint32_t lastPartition,
                     uint32_t* __restrict__ offsets) {
    chained_entry<kChained>();
    __shared__ uint32_t sPart;
    __shared__ uint32_t sScan[kProjectThreads / 32];
    __shared__ unsigned long long sBase;
    const uint32_t tid = threadIdx.x;
    if (tid == 0) sPart = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t part = sPart;
    const uint32_t d0 = (part * kProjectThreads + tid) * kOffsetItems;
    uint32_t slot[kOffsetItems], count[kOffsetItems];
    uint32_t mine = 0;
#pragma unroll
    for (uint32_t k = 0; k < kOffsetItems; ++k) {
        const bool in = d0 + k < n;
        slot[k] = in ? static_cast<uint32_t>(__ldg(sortedWords + d0 + k)) : 0u;
        count[k] = in ? __ldg(touchedIn + slot[k]) : 0u;
        mine += count[k];
    }
    uint32_t blockTotal = 0;
    uint32_t at = block_exclusive_scan(mine, sScan, &blockTotal);
    if (tid < 32) sBase = frame_lookback(status, part, lastPartition, blockTotal, counters, counters + 2);
    __syncthreads();
    const unsigned long long base = sBase;
#pragma unroll
    for (uint32_t k = 0; k < kOffsetItems; ++k) {
        if (d0 + k < n) offsets[slot[k]] = static_cast<uint32_t>(base + at);
        at += count[k];
    }
}

// Block b writes the pairs of slots [256 b, 256 b + 256): it reads each
// one's touched count, rectangle, aux word (project_emit_kernel<.., false>)
// and offset, and, for a splat written row by row or tile by tile, its
// record.
template <bool kChained>
__global__ void __launch_bounds__(kProjectThreads, 4)
emit_pairs_kernel(uint32_t n, const ProjRecord* __restrict__ proj, const uint4* __restrict__ rectsIn,
                  const uint32_t* __restrict__ touchedIn, const unsigned long long* __restrict__ aux,
                  const uint32_t* __restrict__ offsets, uint32_t width, uint32_t height, uint32_t tilesX,
                  uint32_t* __restrict__ err, unsigned long long* __restrict__ pairs, uint32_t capacity,
                  TrainOutputs train, uint32_t* __restrict__ tileDigits, uint32_t tilePasses,
                  const uint2* __restrict__ rowTable) {
    chained_entry<kChained>();
    __shared__ uint32_t sScan[kProjectThreads / 32];
    __shared__ uint32_t sStart[kProjectThreads + 1];
    __shared__ uint32_t sSmallStart[kProjectThreads + 1];
    __shared__ unsigned long long sLow[kProjectThreads];
    __shared__ uint32_t sRect[kProjectThreads];
    __shared__ uint32_t sWidth[kProjectThreads];
    __shared__ Footprint sFoot[kProjectThreads];
    __shared__ uint32_t sFootRow[kProjectThreads + 1];
    __shared__ uint32_t sDigits[2 * 256];
    const uint32_t tid = threadIdx.x;
    sDigits[tid] = 0;
    sDigits[256 + tid] = 0;
    const uint32_t slotBase = blockIdx.x * kProjectThreads;
    const uint32_t slot = slotBase + tid;
    const bool inRange = slot < n;
    const uint32_t touched = inRange ? __ldg(touchedIn + slot) : 0u;
    const bool alive = touched != 0;
    const uint4 rect = alive ? __ldg(rectsIn + slot) : make_uint4(1, 1, 0, 0);
    const uint32_t rw = alive ? rect.z - rect.x + 1 : 0;
    const uint32_t rh = alive ? rect.w - rect.y + 1 : 0;
    const uint32_t area = rw * rh;
    const uint32_t sh = rw <= 1 ? 0u : 32u - static_cast<uint32_t>(__clz(rw - 1));
    const bool masked = alive && area <= kMaskArea;
    const ulonglong2 a = alive ? __ldg(reinterpret_cast<const ulonglong2*>(aux) + slot) : make_ulonglong2(0ull, 0ull);
    const bool irregular = alive && !masked && (a.x & 1ull) != 0;
    // The splats written a row at a time: unmasked, of more than kWarpArea
    // tiles, every row one run. The other unmasked ones go tile by tile.
    const bool rowsHere = alive && !masked && !irregular && area > kWarpArea;
    const bool byWarp = alive && !masked && !rowsHere;
    uint32_t bigTotal = 0, rowsTotal = 0;
    const uint32_t bigIdx = block_exclusive_scan(rowsHere ? 1u : 0u, sScan, &bigTotal);
    const uint32_t rowStart = block_exclusive_scan(rowsHere ? rh : 0u, sScan, &rowsTotal);
    if (rowsHere) {
        const ProjRecord rec = proj[slot];
        sFoot[bigIdx] = Footprint{rec.screen.x, rec.screen.y, rec.conic.x, rec.conic.y, rec.conic.z, rec.screen.w,
                                  rect.x, rect.z, rect.y, tid, static_cast<uint32_t>(a.x >> 32)};
        sFootRow[bigIdx] = rowStart;
    }
    if (tid == 0) sFootRow[bigTotal] = rowsTotal;
    const uint32_t first = alive ? __ldg(offsets + slot) : 0u;
    sStart[tid] = first;
    sLow[tid] = 0ull;
    sRect[tid] = rect.x | (rect.y << 16);
    sWidth[tid] = rw | (sh << 16) | (irregular ? 0x80000000u : 0u);
    __syncthreads();
    const CountingSink sink{PairSink{pairs, train.values, train.emitSlot, capacity, err}, sDigits, tilePasses};
    constexpr uint32_t tileShift = 32;

    // Masked splats: each warp writes its own splats' pairs, 32 at a time,
    // consecutive lanes on consecutive pairs. A lane finds its pair's splat by
    // a binary search over the warp's running pair counts (shuffles: the
    // last lane whose count starts at or before the pair, which always has
    // pairs), and the pair's tile as that splat's mask bit of the same rank.
    {
        const uint32_t lane = tid & 31u;
        const uint32_t mine = masked ? touched : 0u;
        uint32_t incl = mine;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= d) incl += o;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        const uint32_t excl = incl - mine;
        const uint32_t mRect = rect.x | (rect.y << 16);
        const float mInvW = masked ? 1.0f / static_cast<float>(rw) : 0.0f;
        const uint32_t warpBase = slotBase + (tid & ~31u);
        for (uint32_t c0 = 0; c0 < total; c0 += 32) {
            const uint32_t pos = c0 + lane;
            uint32_t l = 0;
#pragma unroll
            for (uint32_t step = 16; step >= 1; step >>= 1) {
                const uint32_t e = __shfl_sync(0xFFFFFFFFu, excl, static_cast<int>(l + step));
                if (e <= pos) l += step;
            }
            const uint32_t r = pos - __shfl_sync(0xFFFFFFFFu, excl, static_cast<int>(l));
            const unsigned long long m = __shfl_sync(0xFFFFFFFFu, a.x, static_cast<int>(l));
            const unsigned long long mH = __shfl_sync(0xFFFFFFFFu, a.y, static_cast<int>(l));
            const uint32_t oRect = __shfl_sync(0xFFFFFFFFu, mRect, static_cast<int>(l));
            const uint32_t oW = __shfl_sync(0xFFFFFFFFu, rw, static_cast<int>(l));
            const float oInvW = __shfl_sync(0xFFFFFFFFu, mInvW, static_cast<int>(l));
            const uint32_t oFirst = __shfl_sync(0xFFFFFFFFu, first, static_cast<int>(l));
            if (pos < total) {
                uint32_t dx, dy;
                mask_bit_tile(nth_set_bit128(m, mH, r), oW, oInvW, dx, dy);
                const uint32_t tx = (oRect & 0xFFFFu) + dx;
                const uint32_t ty = (oRect >> 16) + dy;
                sink.put(static_cast<unsigned long long>(oFirst) + r,
                         static_cast<unsigned long long>(ty * tilesX + tx) << tileShift, warpBase + l);
            }
        }
    }
    if (rowsTotal != 0) {
        uint32_t takenTotal = 0;
        sSmallStart[tid] = block_exclusive_scan(rowsHere ? touched : 0u, sScan, &takenTotal);
        __syncthreads();
        if (takenTotal != 0)
            emit_large_rows(sFoot, sFootRow, bigTotal, rowsTotal, width, height, 0u, tilesX, sWidth, sStart,
                            sSmallStart, sLow, sScan, 0ull, tileShift, slotBase,
                            nullptr, sink, rowTable);
    }
    if (__ballot_sync(0xFFFFFFFFu, byWarp) != 0)
        emit_by_warp(byWarp, area, sWidth, sRect, sStart, sLow, proj + slotBase, width, height, 0u, tilesX, 0ull,
                     tileShift, slotBase, nullptr, sink);
    __syncthreads();
    for (uint32_t d = tid; d < tilePasses * 256; d += kProjectThreads) {
        const uint32_t v = sDigits[d];
        if (v != 0) atomicAdd(tileDigits + d, v);
    }
}

template <class Src>
cudaError_t launch(const FrameParams& f, const FrameParams* fDev, const Src& src, TrainOutputs train, bool stage,
                   ProjRecord* proj, uint4* rects,
                   uint32_t* touched, uint32_t* keys, uint32_t* counters, uint64_t* status, uint32_t* ticket,
                   uint32_t partitionBase, uint32_t lastPartition, uint32_t slotBits, uint64_t* pairs,
                   uint32_t capacity, cudaStream_t stream) {
    const uint32_t stageWords = stage ? f.shWords : 0u;
    const uint32_t shVector = (reinterpret_cast<uintptr_t>(src.sh) & 15u) == 0 ? 1u : 0u;
    const size_t smem = stage ? size_t{kProjectThreads} * f.shWords * 4 : 0;
    cudaError_t e = cudaFuncSetAttribute(project_emit_kernel<Src>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(std::max<size_t>(smem, 1)));
    if (e != cudaSuccess) return e;
    const uint32_t blocks = project_partitions(f.count);
    project_emit_kernel<Src><<<blocks, kProjectThreads, smem, stream>>>(
        f, fDev, src, train, stageWords, shVector, proj, rects, touched, keys, counters, status, ticket, partitionBase,
        lastPartition, slotBits, reinterpret_cast<unsigned long long*>(pairs), capacity);
    return cudaGetLastError();
}

// The projection without its emission (project_emit_kernel<Src, false>).
template <class Src>
cudaError_t launch_only(const FrameParams& f, const Src& src, bool stage, ProjRecord* proj, uint4* rects,
                        uint32_t* touched, uint32_t* keys, uint32_t* counters, uint32_t* ticket, uint64_t* aux,
                        uint64_t* depthWords, uint32_t* depthDigits, uint2* rowTable, uint32_t rowCap,
                        cudaStream_t stream) {
    const uint32_t stageWords = stage ? f.shWords : 0u;
    const uint32_t shVector = (reinterpret_cast<uintptr_t>(src.sh) & 15u) == 0 ? 1u : 0u;
    const size_t smem = stage ? size_t{kProjectThreads} * f.shWords * 4 : 0;
    for (auto kernel : {project_emit_kernel<Src, false, true>, project_emit_kernel<Src, false, false>}) {
        const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(std::max<size_t>(smem, 1)));
        if (e != cudaSuccess) return e;
    }
    const uint32_t blocks = project_partitions(f.count);
    return launch_chained(project_emit_kernel<Src, false, true>, project_emit_kernel<Src, false, false>, dim3(blocks), dim3(kProjectThreads), smem, stream, f,
                          static_cast<const FrameParams*>(nullptr), src, TrainOutputs{nullptr, nullptr, nullptr},
                          stageWords, shVector, proj, rects, touched, keys, counters,
                          static_cast<uint64_t*>(nullptr), ticket, 0u, 0u, 0u, static_cast<unsigned long long*>(nullptr),
                          0u, reinterpret_cast<unsigned long long*>(aux),
                          reinterpret_cast<unsigned long long*>(depthWords), depthDigits, rowTable, rowCap);
}

}  // namespace

size_t project_status_bytes(uint32_t partitions) { return size_t{partitions} * sizeof(uint64_t); }
uint32_t project_partitions(uint32_t count) { return (count + kProjectThreads - 1) / kProjectThreads; }

cudaError_t launch_project_emit(const FrameParams& f, const float4* positions, const uint4* shape, const uint32_t* sh,
                                ProjRecord* proj, uint4* rects, uint32_t* touched, uint32_t* keys, uint32_t* counters,
                                uint64_t* status, uint32_t* ticket, uint32_t partitionBase, uint32_t lastPartition,
                                uint32_t slotBits, uint64_t* pairs, uint32_t capacity, cudaStream_t stream,
                                const FrameParams* fDev, const float* filter3d) {
    if (f.count == 0) return cudaSuccess;
    const uint32_t rpc = f.restPerColour;
    const uint32_t stored = rpc >= 15 ? 3u : rpc >= 8 ? 2u : rpc >= 3 ? 1u : 0u;
    const bool stage = std::min(stored, f.shLimit) > 0 && f.shWords > 0;
    return launch(f, fDev, PackedSource{positions, shape, sh, filter3d}, TrainOutputs{nullptr, nullptr, nullptr}, stage,
                  proj, rects,
                  touched, keys, counters, status, ticket, partitionBase, lastPartition, slotBits, pairs, capacity,
                  stream);
}

cudaError_t launch_project_points(const FrameParams& f, const float4* positions, const uint32_t* colours,
                                  const lrt_point_style& style, ProjRecord* proj, uint4* rects, uint32_t* touched,
                                  uint32_t* keys, uint32_t* counters, uint64_t* status, uint32_t* ticket,
                                  uint32_t partitionBase, uint32_t lastPartition, uint32_t slotBits, uint64_t* pairs,
                                  uint32_t capacity, cudaStream_t stream) {
    if (f.count == 0) return cudaSuccess;
    PointSource src{positions, reinterpret_cast<const uint2*>(colours), nullptr, style.size_mode, style.size,
                    style.constant_colour, {style.colour[0], style.colour[1], style.colour[2]}};
    return launch(f, nullptr, src, TrainOutputs{nullptr, nullptr, nullptr}, false, proj, rects, touched, keys,
                  counters, status, ticket, partitionBase, lastPartition, slotBits, pairs, capacity, stream);
}

cudaError_t launch_project_emit_train(const FrameParams& f, const float* means, const float* logScales,
                                      const float* quats, const float* logits, const uint16_t* sh, ProjRecord* proj,
                                      uint4* rects, uint32_t* touched, uint32_t* keys, uint32_t* offsets,
                                      uint32_t* counters, uint64_t* status, uint32_t* ticket, uint32_t partitionBase,
                                      uint32_t lastPartition, uint32_t lowBits, uint64_t* pairs, uint32_t* values,
                                      uint32_t* emitSlot, uint32_t capacity, cudaStream_t stream,
                                      const FrameParams* fDev) {
    if (f.count == 0) return cudaSuccess;
    // The DC triple is read from the staged row too, so it is always staged.
    return launch(f, fDev, RawSource{means, logScales, quats, logits, reinterpret_cast<const uint32_t*>(sh)},
                  TrainOutputs{offsets, values, emitSlot}, true, proj, rects, touched, keys, counters, status, ticket,
                  partitionBase, lastPartition, lowBits, pairs, capacity, stream);
}

cudaError_t launch_project_only(const FrameParams& f, const float4* positions, const uint4* shape, const uint32_t* sh,
                                const float* filter3d, ProjRecord* proj, uint4* rects, uint32_t* touched,
                                uint32_t* keys, uint32_t* counters, uint32_t* ticket, uint64_t* aux,
                                uint64_t* depthWords, uint32_t* depthDigits,
                                uint2* rowTable, uint32_t rowCap, cudaStream_t stream) {
    if (f.count == 0) return cudaSuccess;
    const uint32_t rpc = f.restPerColour;
    const uint32_t stored = rpc >= 15 ? 3u : rpc >= 8 ? 2u : rpc >= 3 ? 1u : 0u;
    const bool stage = std::min(stored, f.shLimit) > 0 && f.shWords > 0;
    return launch_only(f, PackedSource{positions, shape, sh, filter3d}, stage, proj, rects, touched, keys, counters,
                       ticket, aux, depthWords, depthDigits, rowTable, rowCap, stream);
}

cudaError_t launch_project_points_only(const FrameParams& f, const float4* positions, const uint32_t* colours,
                                       const lrt_point_style& style, ProjRecord* proj, uint4* rects, uint32_t* touched,
                                       uint32_t* keys, uint32_t* counters, uint32_t* ticket, uint64_t* aux,
                                       uint64_t* depthWords, uint32_t* depthDigits,
                                uint2* rowTable, uint32_t rowCap, cudaStream_t stream) {
    if (f.count == 0) return cudaSuccess;
    PointSource src{positions, reinterpret_cast<const uint2*>(colours), nullptr, style.size_mode, style.size,
                    style.constant_colour, {style.colour[0], style.colour[1], style.colour[2]}};
    return launch_only(f, src, false, proj, rects, touched, keys, counters, ticket, aux, depthWords, depthDigits,
                       rowTable, rowCap, stream);
}

cudaError_t launch_emit_sorted(const uint64_t* sortedWords, uint32_t n, const ProjRecord* proj, const uint4* rects,
                               const uint32_t* touched, const uint64_t* aux, uint32_t width, uint32_t height,
                               uint32_t tilesX, uint32_t* counters, uint64_t* status, uint32_t* ticket,
                               uint32_t* offsets, uint64_t* pairs, uint32_t capacity, uint32_t* tileDigits,
                               uint32_t tilePasses, const uint2* rowTable, cudaStream_t stream, uint32_t* values,
                               uint32_t* emitSlot) {
    if (n == 0) return cudaSuccess;
    const uint32_t perBlock = kProjectThreads * kOffsetItems;
    const uint32_t offsetBlocks = (n + perBlock - 1) / perBlock;
    cudaError_t e = launch_chained(depth_offsets_kernel<true>, depth_offsets_kernel<false>, dim3(offsetBlocks), dim3(kProjectThreads), 0, stream,
                                   reinterpret_cast<const unsigned long long*>(sortedWords), n, touched, counters,
                                   status, ticket, offsetBlocks - 1, offsets);
    if (e != cudaSuccess) return e;
    return launch_chained(emit_pairs_kernel<true>, emit_pairs_kernel<false>, dim3(project_partitions(n)), dim3(kProjectThreads), 0, stream, n, proj,
                          rects, touched, reinterpret_cast<const unsigned long long*>(aux),
                          static_cast<const uint32_t*>(offsets), width, height, tilesX, counters + 2,
                          reinterpret_cast<unsigned long long*>(pairs), capacity,
                          TrainOutputs{nullptr, values, emitSlot}, tileDigits, tilePasses, rowTable);
}

cudaError_t launch_project_only_train(const FrameParams& f, const float* means, const float* logScales,
                                      const float* quats, const float* logits, const uint16_t* sh, ProjRecord* proj,
                                      uint4* rects, uint32_t* touched, uint32_t* keys, uint32_t* counters,
                                      uint32_t* ticket, uint64_t* aux, uint64_t* depthWords, uint32_t* depthDigits,
                                uint2* rowTable, uint32_t rowCap, cudaStream_t stream) {
    if (f.count == 0) return cudaSuccess;
    // The DC triple is read from the staged row too, so it is always staged.
    return launch_only(f, RawSource{means, logScales, quats, logits, reinterpret_cast<const uint32_t*>(sh)}, true,
                       proj, rects, touched, keys, counters, ticket, aux, depthWords, depthDigits, rowTable, rowCap,
                       stream);
}

}  // namespace lrt
