// ORACLE -- test infrastructure, not product code. See lrt_oracle.h.
//
// Compile with -ffp-contract=off and without -ffast-math: every float
// expression below is evaluated in the order written, one rounding per
// operation, which is the contract the product's kernels (built with
// -fmad=false) are checked against bit for bit.
#include "lrt_oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <thread>
#include <vector>

namespace {

constexpr uint32_t kTile = 16;   // shaders/lrt/splat/frame.slang:31

// ----------------------------------------------------------------- bits ---
inline uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float bitsf(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// --------------------------------------------------- exp / log / pow -------
// Our own, not the C library's: the product computes the same functions with
// the same method on the device, so both sides round identically.
//
// exp: Cody & Waite argument reduction, x = n ln2 + r with n = rint(x log2 e)
// and the reduction done by two fused multiply-adds with ln 2 split into a
// float and its float remainder; e^r from its Taylor series to degree 7
// (Horner, fused multiply-adds; truncation below 0.2 ulp for |r| <= ln2/2);
// 2^n applied through the exponent field in at most two exact steps and one
// final rounding (which also gives the subnormal range).
constexpr float kLog2e = 1.44269504088896340736f;
constexpr float kLn2Hi = 0.693147182464599609375f;      // (float) ln 2
constexpr float kLn2Lo = -1.904654299957768e-09f;       // (float)(ln 2 - kLn2Hi)

float expImpl(float x) {
    if (x != x) return x;
    if (x > 89.0f) return INFINITY;
    if (x < -104.0f) return 0.0f;
    const float n = std::rint(x * kLog2e);
    float r = std::fma(-n, kLn2Hi, x);
    r = std::fma(-n, kLn2Lo, r);
    float p = 1.984126984126984e-4f;                  // 1/7!
    p = std::fma(p, r, 1.388888888888889e-3f);        // 1/6!
    p = std::fma(p, r, 8.333333333333333e-3f);        // 1/5!
    p = std::fma(p, r, 4.166666666666666e-2f);        // 1/4!
    p = std::fma(p, r, 1.666666666666667e-1f);        // 1/3!
    p = std::fma(p, r, 0.5f);
    p = std::fma(p, r, 1.0f);
    p = std::fma(p, r, 1.0f);
    int e = static_cast<int>(n);
    if (e > 126) {
        p = p * bitsf(253u << 23);   // 2^126
        e -= 126;
    } else if (e < -125) {
        p = p * bitsf(2u << 23);     // 2^-125
        e += 125;
    }
    return p * bitsf(static_cast<uint32_t>(e + 127) << 23);
}

// log: x = m 2^e with m in [sqrt(1/2), sqrt 2]; log m = 2 artanh(s) with
// s = (m - 1)/(m + 1), the artanh series s + s^3/3 + ... + s^11/11 (|s| <=
// 0.172, truncation below 1e-11 relative); e ln 2 added with the split ln 2.
float logImpl(float x) {
    if (x != x) return x;
    if (x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (x == INFINITY) return x;
    int e = 0;
    uint32_t u = fbits(x);
    if (u < 0x00800000u) {
        x = x * 8388608.0f;   // 2^23, exact
        u = fbits(x);
        e = -23;
    }
    e += static_cast<int>(u >> 23) - 127;
    float m = bitsf((u & 0x007FFFFFu) | 0x3F800000u);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float z = s * s;
    float p = std::fma(z, 0.0909090909090909f, 0.1111111111111111f);   // 1/11, 1/9
    p = std::fma(p, z, 0.1428571428571429f);                            // 1/7
    p = std::fma(p, z, 0.2f);                                           // 1/5
    p = std::fma(p, z, 0.3333333333333333f);                            // 1/3
    const float t = 2.0f * s;
    const float lm = std::fma(t * z, p, t);
    const float fe = static_cast<float>(e);
    return std::fma(fe, kLn2Hi, std::fma(fe, kLn2Lo, lm));
}

float powImpl(float x, float y) { return expImpl(y * logImpl(x)); }

// ----------------------------------------------------------------- f16 ----
float halfToFloat(uint32_t h) {
    const uint32_t sign = (h >> 15) & 1u;
    const uint32_t exp = (h >> 10) & 0x1Fu;
    const uint32_t mant = h & 0x3FFu;
    float v;
    if (exp == 0) {
        v = static_cast<float>(mant) * 5.9604644775390625e-08f;   // 2^-24
    } else if (exp == 31) {
        v = mant == 0 ? INFINITY : NAN;
    } else {
        v = bitsf(((exp - 15 + 127) << 23) | (mant << 13));
    }
    return sign ? -v : v;
}

uint32_t floatToHalf(float f) {   // round to nearest, ties to even
    const uint32_t u = fbits(f);
    const uint32_t sign = (u >> 16) & 0x8000u;
    const uint32_t a = u & 0x7FFFFFFFu;
    if (a >= 0x7F800000u) return sign | (a > 0x7F800000u ? 0x7E00u : 0x7C00u);
    if (a >= 0x477FF000u) return sign | 0x7C00u;
    if (a < 0x38800000u) {
        const float v = bitsf(a) * 16777216.0f;   // in units of 2^-24, exact
        return sign | static_cast<uint32_t>(std::rint(v));
    }
    const uint32_t mant = a & 0x7FFFFFu;
    uint32_t h = ((((a >> 23) - 127 + 15)) << 10) | (mant >> 13);
    const uint32_t rem = mant & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1;
    return sign | h;
}

inline float lowHalf(uint32_t w) { return halfToFloat(w & 0xFFFFu); }   // packing.slang:108
inline float highHalf(uint32_t w) { return halfToFloat(w >> 16); }      // packing.slang:109

// ------------------------------------------------------------ float3 -------
struct F3 {
    float x, y, z;
};
inline float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 normalize3(F3 v) {
    const float l = std::sqrt(dot3(v, v));
    return {v.x / l, v.y / l, v.z / l};
}
inline float clampf(float v, float lo, float hi) { return std::fmin(std::fmax(v, lo), hi); }
inline float saturatef(float v) { return clampf(v, 0.0f, 1.0f); }

// ------------------------------------------------------------ camera -------
// modules/aofx/sdk/include/aofx/Transform.h and modules/render/src/Camera.cpp.
struct M4 {
    double m[16];
    double at(int r, int c) const { return m[r * 4 + c]; }
    double& at(int r, int c) { return m[r * 4 + c]; }
    static M4 identity() {
        M4 o{};
        o.m[0] = o.m[5] = o.m[10] = o.m[15] = 1.0;
        return o;
    }
};
M4 mul4(const M4& a, const M4& b) {   // Transform.h:97-109
    M4 o{};
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += a.at(r, k) * b.at(k, c);
            o.at(r, c) = s;
        }
    return o;
}
struct D3 {
    double x, y, z;
};
D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
D3 scale(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double dotd(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
D3 crossd(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double lengthd(D3 a) { return std::sqrt(dotd(a, a)); }
D3 normalisedd(D3 a) {
    const double l = lengthd(a);
    return l > 1e-12 ? scale(a, 1.0 / l) : D3{0, 0, 0};
}
D3 pointOf(const M4& m, D3 p) {   // Transform.h:72-76
    return {m.at(0, 0) * p.x + m.at(0, 1) * p.y + m.at(0, 2) * p.z + m.at(0, 3),
            m.at(1, 0) * p.x + m.at(1, 1) * p.y + m.at(1, 2) * p.z + m.at(1, 3),
            m.at(2, 0) * p.x + m.at(2, 1) * p.y + m.at(2, 2) * p.z + m.at(2, 3)};
}
M4 inverseAffine(const M4& m) {   // Transform.h:334-361
    const double a00 = m.at(0, 0), a01 = m.at(0, 1), a02 = m.at(0, 2);
    const double a10 = m.at(1, 0), a11 = m.at(1, 1), a12 = m.at(1, 2);
    const double a20 = m.at(2, 0), a21 = m.at(2, 1), a22 = m.at(2, 2);
    const double c00 = a11 * a22 - a12 * a21;
    const double c01 = a12 * a20 - a10 * a22;
    const double c02 = a10 * a21 - a11 * a20;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    const double inv = std::fabs(det) > 1e-18 ? 1.0 / det : 0.0;
    M4 o = M4::identity();
    o.at(0, 0) = c00 * inv;
    o.at(0, 1) = (a02 * a21 - a01 * a22) * inv;
    o.at(0, 2) = (a01 * a12 - a02 * a11) * inv;
    o.at(1, 0) = c01 * inv;
    o.at(1, 1) = (a00 * a22 - a02 * a20) * inv;
    o.at(1, 2) = (a02 * a10 - a00 * a12) * inv;
    o.at(2, 0) = c02 * inv;
    o.at(2, 1) = (a01 * a20 - a00 * a21) * inv;
    o.at(2, 2) = (a00 * a11 - a01 * a10) * inv;
    const D3 t{m.at(0, 3), m.at(1, 3), m.at(2, 3)};
    const D3 back{-(o.at(0, 0) * t.x + o.at(0, 1) * t.y + o.at(0, 2) * t.z),
                  -(o.at(1, 0) * t.x + o.at(1, 1) * t.y + o.at(1, 2) * t.z),
                  -(o.at(2, 0) * t.x + o.at(2, 1) * t.y + o.at(2, 2) * t.z)};
    o.at(0, 3) = back.x;
    o.at(1, 3) = back.y;
    o.at(2, 3) = back.z;
    return o;
}

M4 toM4(const double* m) {
    M4 o;
    std::memcpy(o.m, m, sizeof(o.m));
    return o;
}

// ------------------------------------------------------------- edit --------
// shaders/lrt/common/edit.slang:23-85.
struct Fate {
    bool removed, graded;
    float opacity;
};
Fate editFate(const lrt_splat_edit& e, F3 p, float opacity, F3 s) {
    Fate f{false, false, opacity};
    if (e.active == 0) return f;
    if (e.min_opacity > 0.0f && opacity < e.min_opacity) {
        f.removed = true;
        return f;
    }
    if (e.max_scale > 0.0f &&
        std::fmax(std::fmax(std::fabs(s.x), std::fabs(s.y)), std::fabs(s.z)) > e.max_scale) {
        f.removed = true;
        return f;
    }
    const F3 rel{p.x - e.centre[0], p.y - e.centre[1], p.z - e.centre[2]};
    bool inside = e.shape == 1 ? dot3(rel, rel) <= e.size[0] * e.size[0]
                               : (std::fabs(rel.x) <= e.size[0] && std::fabs(rel.y) <= e.size[1] &&
                                  std::fabs(rel.z) <= e.size[2]);
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
F3 editGrade(const lrt_splat_edit& e, F3 c0) {
    const F3 c{c0.x * e.tint[0] * e.brightness, c0.y * e.tint[1] * e.brightness,
               c0.z * e.tint[2] * e.brightness};
    const float luma = dot3(c, F3{0.2126f, 0.7152f, 0.0722f});
    // lerp(a, b, t) = a + (b - a) * t
    return {std::fmax(luma + (c.x - luma) * e.saturation, 0.0f),
            std::fmax(luma + (c.y - luma) * e.saturation, 0.0f),
            std::fmax(luma + (c.z - luma) * e.saturation, 0.0f)};
}

// -------------------------------------------------------------- frame ------
// shaders/lrt/splat/frame.slang:33-81 (the fields the raster reads).
struct Frame {
    uint32_t width, height, tilesX, tilesY;
    float focalX, focalY, centreX, centreY, nearZ, farZ;
    uint32_t ortho, antialias;
    float m[12];
    float eye[3];
    uint32_t count, base, restPerColour, shWords, shLimit;
    uint32_t depthMode;
    float depthThreshold;
    float bg[4];
    uint32_t linearise;
    lrt_splat_edit edit;
};

Frame frameFor(const lrt_projection& pr, const lrt_render_settings& s) {   // FrameParams.h:32-56
    Frame f{};
    f.width = s.width;
    f.height = s.height;
    f.tilesX = (s.width + kTile - 1) / kTile;
    f.tilesY = (s.height + kTile - 1) / kTile;
    f.focalX = static_cast<float>(pr.focal_x);
    f.focalY = static_cast<float>(pr.focal_y);
    f.centreX = static_cast<float>(pr.centre_x);
    f.centreY = static_cast<float>(pr.centre_y);
    f.nearZ = static_cast<float>(pr.near_z);
    f.farZ = static_cast<float>(pr.far_z);
    f.ortho = pr.orthographic ? 1u : 0u;
    f.antialias = s.antialias ? 1u : 0u;
    f.shLimit = s.max_sh_degree;
    f.depthMode = s.depth_mode;
    f.depthThreshold = s.depth_threshold;
    for (int k = 0; k < 4; ++k) f.bg[k] = s.background[k];
    f.linearise = s.linearise ? 1u : 0u;
    return f;
}

void setObject(Frame& f, const lrt_projection& pr, const lrt_splat_instance& inst) {
    // TileRasterizer.cpp:297-299 and FrameParams.h:58-69
    const M4 toWorld = toM4(inst.object_to_world);
    const M4 objectToView = mul4(toM4(pr.world_to_view), toWorld);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) f.m[r * 4 + c] = static_cast<float>(objectToView.at(r, c));
    const D3 eye = pointOf(inverseAffine(toWorld), D3{pr.eye_world[0], pr.eye_world[1], pr.eye_world[2]});
    f.eye[0] = static_cast<float>(eye.x);
    f.eye[1] = static_cast<float>(eye.y);
    f.eye[2] = static_cast<float>(eye.z);
    f.edit = inst.edit;
}

F3 toView(const Frame& f, F3 p) {   // frame.slang:91-95
    return {f.m[0] * p.x + f.m[1] * p.y + f.m[2] * p.z + f.m[3],
            f.m[4] * p.x + f.m[5] * p.y + f.m[6] * p.z + f.m[7],
            f.m[8] * p.x + f.m[9] * p.y + f.m[10] * p.z + f.m[11]};
}

float cutoffPower(float alpha) {   // frame.slang:105-107
    return std::fmin(2.0f * logImpl(std::fmax(255.0f * alpha, 1.0001f)), 9.0f);
}

float minPowerOverBox(float a, float b, float c, float lox, float loy, float hix, float hiy) {
    // frame.slang:113-130
    if (lox <= 0.0f && hix >= 0.0f && loy <= 0.0f && hiy >= 0.0f) return 0.0f;
    float best = 3.4e38f;
    for (int e = 0; e < 2; ++e) {
        const float x = e == 0 ? lox : hix;
        const float y = c > 1e-12f ? clampf(-b * x / c, loy, hiy) : loy;
        best = std::fmin(best, a * x * x + 2.0f * b * x * y + c * y * y);
    }
    for (int e = 0; e < 2; ++e) {
        const float y = e == 0 ? loy : hiy;
        const float x = a > 1e-12f ? clampf(-b * y / a, lox, hix) : lox;
        best = std::fmin(best, a * x * x + 2.0f * b * x * y + c * y * y);
    }
    return best;
}

bool tileTouched(const Frame& f, float cx, float cy, F3 conic, float cutoff, uint32_t tx,
                 uint32_t ty) {   // frame.slang:133-138
    const float firstX = static_cast<float>(tx * kTile) + 0.5f;
    const float firstY = static_cast<float>(ty * kTile) + 0.5f;
    const float lastX = static_cast<float>(std::min((tx + 1) * kTile, f.width) - 1) + 0.5f;
    const float lastY = static_cast<float>(std::min((ty + 1) * kTile, f.height) - 1) + 0.5f;
    return minPowerOverBox(conic.x, conic.y, conic.z, firstX - cx, firstY - cy, lastX - cx,
                           lastY - cy) <= cutoff;
}

struct Rect {
    uint32_t x0, y0, x1, y1;
};
Rect tileRect(const Frame& f, float cx, float cy, float ex, float ey) {   // frame.slang:149-161
    const float x1 = cx - ex;
    const float y1 = cy - ey;
    const float x2 = cx + ex;
    const float y2 = cy + ey;
    if (x2 < 0.0f || y2 < 0.0f || x1 >= static_cast<float>(f.width) ||
        y1 >= static_cast<float>(f.height)) {
        return {1, 1, 0, 0};
    }
    return {static_cast<uint32_t>(std::fmax(x1, 0.0f)) / kTile,
            static_cast<uint32_t>(std::fmax(y1, 0.0f)) / kTile,
            static_cast<uint32_t>(std::fmin(x2, static_cast<float>(f.width) - 1.0f)) / kTile,
            static_cast<uint32_t>(std::fmin(y2, static_cast<float>(f.height) - 1.0f)) / kTile};
}

// ------------------------------------------------------------ packing ------
// shaders/lrt/common/packing.slang:52-69
void decodeQuaternion(uint32_t word, float q[4]) {
    const uint32_t largest = word & 3u;
    float sx = static_cast<float>((word >> 22) & 1023u);
    float sy = static_cast<float>((word >> 12) & 1023u);
    float sz = static_cast<float>((word >> 2) & 1023u);
    sx = (sx / 1023.0f * 2.0f - 1.0f) * 0.70710678f;
    sy = (sy / 1023.0f * 2.0f - 1.0f) * 0.70710678f;
    sz = (sz / 1023.0f * 2.0f - 1.0f) * 0.70710678f;
    const float small[3] = {sx, sy, sz};
    const float rest = std::sqrt(std::fmax(0.0f, 1.0f - (sx * sx + sy * sy + sz * sz)));
    uint32_t next = 0;
    for (uint32_t k = 0; k < 4; ++k) {
        if (k == largest) {
            q[k] = rest;
        } else {
            q[k] = small[next++];
        }
    }
}

// packing.slang:26-50
uint32_t encodeQuaternion(const float q0[4]) {
    const float l = std::sqrt(q0[0] * q0[0] + q0[1] * q0[1] + q0[2] * q0[2] + q0[3] * q0[3]);
    float q[4] = {q0[0] / l, q0[1] / l, q0[2] / l, q0[3] / l};
    uint32_t largest = 0;
    float best = std::fabs(q[0]);
    for (uint32_t k = 1; k < 4; ++k) {
        if (std::fabs(q[k]) > best) {
            best = std::fabs(q[k]);
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
        const float unit = clampf(q[k] / 0.70710678f * 0.5f + 0.5f, 0.0f, 1.0f);
        word |= static_cast<uint32_t>(std::round(unit * 1023.0f)) << shift;
        shift -= 10;
    }
    return word;
}

inline float halfSafe(float v) { return clampf(v, -65000.0f, 65000.0f); }   // packing.slang:113
inline uint32_t packHalves(float a, float b) {                              // packing.slang:104-106
    return (floatToHalf(a) & 0xFFFFu) | ((floatToHalf(b) & 0xFFFFu) << 16);
}
constexpr float kSH0 = 0.28209479177387814f;

// ----------------------------------------------------------------- SH -------
// shaders/lrt/common/sh.slang:8-51
constexpr float kC1 = 0.4886025119029199f;
constexpr float kC2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                          -1.0925484305920792f, 0.5462742152960396f};
constexpr float kC3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                          0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                          -0.5900435899266435f};

inline float halfAt(const uint32_t* row, uint32_t index) {
    const uint32_t w = row[index / 2];
    return (index & 1u) == 0u ? lowHalf(w) : highHalf(w);
}
inline F3 basisAt(const uint32_t* row, uint32_t off, uint32_t k) {
    return {halfAt(row, off + k * 3), halfAt(row, off + k * 3 + 1), halfAt(row, off + k * 3 + 2)};
}
uint32_t degreeOf(uint32_t rest) { return rest >= 15 ? 3 : rest >= 8 ? 2 : rest >= 3 ? 1 : 0; }

// `off`: where the rest coefficients start in the row, in halves (0 in the
// packed layout; 3, after the DC triple, in the training layout).
F3 evaluateRest(const uint32_t* row, uint32_t degree, F3 dir, uint32_t off = 0) {
    auto basis = [&](const uint32_t* rw, uint32_t k) { return basisAt(rw, off, k); };
    if (degree == 0) return {0.0f, 0.0f, 0.0f};
    const float x = dir.x, y = dir.y, z = dir.z;
    const float s0 = -kC1 * y, s1 = kC1 * z, s2 = kC1 * x;
    const F3 b0 = basis(row, 0), b1 = basis(row, 1), b2 = basis(row, 2);
    F3 r{s0 * b0.x + s1 * b1.x - s2 * b2.x, s0 * b0.y + s1 * b1.y - s2 * b2.y,
         s0 * b0.z + s1 * b1.z - s2 * b2.z};
    if (degree < 2) return r;
    const float xx = x * x, yy = y * y, zz = z * z;
    const float xy = x * y, yz = y * z, xz = x * z;
    {
        const float t0 = kC2[0] * xy, t1 = kC2[1] * yz, t2 = kC2[2] * (2.0f * zz - xx - yy),
                    t3 = kC2[3] * xz, t4 = kC2[4] * (xx - yy);
        const F3 b3 = basis(row, 3), b4 = basis(row, 4), b5 = basis(row, 5), b6 = basis(row, 6),
                 b7 = basis(row, 7);
        r.x = r.x + (t0 * b3.x + t1 * b4.x + t2 * b5.x + t3 * b6.x + t4 * b7.x);
        r.y = r.y + (t0 * b3.y + t1 * b4.y + t2 * b5.y + t3 * b6.y + t4 * b7.y);
        r.z = r.z + (t0 * b3.z + t1 * b4.z + t2 * b5.z + t3 * b6.z + t4 * b7.z);
    }
    if (degree < 3) return r;
    {
        const float t0 = kC3[0] * y * (3.0f * xx - yy), t1 = kC3[1] * xy * z,
                    t2 = kC3[2] * y * (4.0f * zz - xx - yy),
                    t3 = kC3[3] * z * (2.0f * zz - 3.0f * xx - 3.0f * yy),
                    t4 = kC3[4] * x * (4.0f * zz - xx - yy), t5 = kC3[5] * z * (xx - yy),
                    t6 = kC3[6] * x * (xx - 3.0f * yy);
        const F3 b8 = basis(row, 8), b9 = basis(row, 9), b10 = basis(row, 10),
                 b11 = basis(row, 11), b12 = basis(row, 12), b13 = basis(row, 13),
                 b14 = basis(row, 14);
        r.x = r.x + (t0 * b8.x + t1 * b9.x + t2 * b10.x + t3 * b11.x + t4 * b12.x + t5 * b13.x +
                     t6 * b14.x);
        r.y = r.y + (t0 * b8.y + t1 * b9.y + t2 * b10.y + t3 * b11.y + t4 * b12.y + t5 * b13.y +
                     t6 * b14.y);
        r.z = r.z + (t0 * b8.z + t1 * b9.z + t2 * b10.z + t3 * b11.z + t4 * b12.z + t5 * b13.z +
                     t6 * b14.z);
    }
    return r;
}

// -------------------------------------------------------------- colour -----
float srgbToLinear(float c) {   // shaders/lrt/common/color.slang:7-10
    c = std::fmax(c, 0.0f);
    return c <= 0.04045f ? c / 12.92f : powImpl((c + 0.055f) / 1.055f, 2.4f);
}

// ----------------------------------------------------------- threads -------
void parallelFor(uint64_t n, uint32_t threads, const std::function<void(uint64_t, uint64_t)>& fn) {
    if (threads <= 1 || n < 2048) {
        fn(0, n);
        return;
    }
    const uint64_t chunks = std::min<uint64_t>(n, uint64_t{threads} * 16);
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < threads; ++t) {
        pool.emplace_back([&] {
            for (;;) {
                const uint64_t c = next.fetch_add(1);
                if (c >= chunks) return;
                fn(n * c / chunks, n * (c + 1) / chunks);
            }
        });
    }
    for (auto& t : pool) t.join();
}

using Clock = std::chrono::steady_clock;
double msSince(Clock::time_point& t) {
    const auto now = Clock::now();
    const double ms = std::chrono::duration<double, std::milli>(now - t).count();
    t = now;
    return ms;
}

// ---------------------------------------------------------- projection -----
struct Record {
    float screen[4];   // centre.xy, view z, cutoff
    float conic[4];    // a, b, c, alpha
    float colour[4];   // rgb, 0
};

struct Projected {
    std::vector<Record> proj;
    std::vector<Rect> rects;
    std::vector<uint32_t> touched, visible, keys;
};

// Where a splat's parameters come from: the packed cloud (decoded as
// splat_project.slang does) or the training path's raw parameters (means,
// log-scales, quaternions w x y z normalised here, opacity logits, SH fp16
// [16][3] with the DC first: scale exp(log-scale), opacity
// 1 / (1 + exp(-logit)), base colour 0.5 + SH0 * DC).
struct PackedSrc {
    const lrt_gpu_splats& c;
    void load(uint32_t i, F3& p, float& opacity, F3& scale) const {
        const float* pos = static_cast<const float*>(c.positions) + size_t{i} * 4;
        const uint32_t* shape = static_cast<const uint32_t*>(c.shape) + size_t{i} * 4;
        p = {pos[0], pos[1], pos[2]};
        opacity = pos[3];
        scale = {expImpl(lowHalf(shape[1])), expImpl(highHalf(shape[1])), expImpl(lowHalf(shape[2]))};
        if (c.filter3d != nullptr) {
            // The Mip-Splatting 3D filter (Yu et al., CVPR 2024, section 4.1):
            // scales sqrt(s^2 + v), opacity times sqrt(prod s^2 / prod (s^2 + v)).
            const float v = static_cast<const float*>(c.filter3d)[i];
            const float qx = scale.x * scale.x, qy = scale.y * scale.y, qz = scale.z * scale.z;
            const float fx = qx + v, fy = qy + v, fz = qz + v;
            const float before = qx * qy * qz;
            const float after = fx * fy * fz;
            opacity = opacity * std::sqrt(before / after);
            scale = {std::sqrt(fx), std::sqrt(fy), std::sqrt(fz)};
        }
    }
    void rotation(uint32_t i, float q[4]) const {
        decodeQuaternion(static_cast<const uint32_t*>(c.shape)[size_t{i} * 4], q);
    }
    F3 base(uint32_t i) const {
        const uint32_t* shape = static_cast<const uint32_t*>(c.shape) + size_t{i} * 4;
        return {highHalf(shape[2]), lowHalf(shape[3]), highHalf(shape[3])};
    }
    const uint32_t* shRow(uint32_t i) const { return static_cast<const uint32_t*>(c.sh) + size_t{i} * c.sh_words; }
    uint32_t restOffset() const { return 0; }
    uint32_t restPerColour() const { return c.rest_per_colour; }
};

struct RawSrc {
    const lrt_train_params& t;
    void load(uint32_t i, F3& p, float& opacity, F3& scale) const {
        const float* m = static_cast<const float*>(t.means) + size_t{i} * 3;
        const float* ls = static_cast<const float*>(t.log_scales) + size_t{i} * 3;
        p = {m[0], m[1], m[2]};
        opacity = 1.0f / (1.0f + expImpl(-static_cast<const float*>(t.opacity_logits)[i]));
        scale = {expImpl(ls[0]), expImpl(ls[1]), expImpl(ls[2])};
    }
    void rotation(uint32_t i, float q[4]) const {
        const float* r = static_cast<const float*>(t.quats) + size_t{i} * 4;   // w x y z
        const float len = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
        if (len > 0.0f) {
            q[0] = r[1] / len;
            q[1] = r[2] / len;
            q[2] = r[3] / len;
            q[3] = r[0] / len;
        } else {
            q[0] = q[1] = q[2] = 0.0f;
            q[3] = 1.0f;
        }
    }
    F3 base(uint32_t i) const {
        const uint32_t* row = shRow(i);
        return {0.5f + kSH0 * halfAt(row, 0), 0.5f + kSH0 * halfAt(row, 1), 0.5f + kSH0 * halfAt(row, 2)};
    }
    const uint32_t* shRow(uint32_t i) const { return static_cast<const uint32_t*>(t.sh) + size_t{i} * 24; }
    uint32_t restOffset() const { return 3; }
    uint32_t restPerColour() const { return 15; }
};

// shaders/lrt/splat/splat_project.slang:39-221 (relight excluded: off in
// every configuration this build serves).
template <class Src>
void projectOne(const Frame& f, const Src& src, uint32_t i, Projected& out) {
    const uint32_t slot = f.base + i;
    auto cull = [&] {
        out.touched[slot] = 0;
        out.visible[slot] = 0;
        out.keys[slot] = 0x00FFFFFFu;
        out.rects[slot] = {1, 1, 0, 0};
        out.proj[slot] = Record{};
    };
    F3 p, scale;
    float opacity;
    src.load(i, p, opacity, scale);
    const Fate fate = editFate(f.edit, p, opacity, scale);
    if (fate.removed) return cull();
    opacity = fate.opacity;

    const F3 t = toView(f, p);
    if (!(t.z > f.nearZ) || t.z > f.farZ) return cull();

    float q[4];
    src.rotation(i, q);
    const float x = q[0], y = q[1], z = q[2], w = q[3];
    const float r[3][3] = {
        {1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y - w * z), 2.0f * (x * z + w * y)},
        {2.0f * (x * y + w * z), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z - w * x)},
        {2.0f * (x * z - w * y), 2.0f * (y * z + w * x), 1.0f - 2.0f * (x * x + y * y)}};
    const float sc[3] = {scale.x, scale.y, scale.z};
    float m[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) m[a][b] = r[a][b] * sc[b];

    float jx[3], jy[3];
    float cx, cy;
    if (f.ortho) {
        jx[0] = f.focalX; jx[1] = 0.0f; jx[2] = 0.0f;
        jy[0] = 0.0f; jy[1] = f.focalY; jy[2] = 0.0f;
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
        jx[0] = f.focalX * invZ; jx[1] = 0.0f; jx[2] = -f.focalX * tx * invZ * invZ;
        jy[0] = 0.0f; jy[1] = f.focalY * invZ; jy[2] = -f.focalY * ty * invZ * invZ;
    }
    // mul(row, matrix): result[j] = row[0] W[0][j] + row[1] W[1][j] + row[2] W[2][j]
    const float wv[3][3] = {{f.m[0], f.m[1], f.m[2]}, {f.m[4], f.m[5], f.m[6]}, {f.m[8], f.m[9], f.m[10]}};
    float tx3[3], ty3[3], ax[3], ay[3];
    for (int j = 0; j < 3; ++j) {
        tx3[j] = jx[0] * wv[0][j] + jx[1] * wv[1][j] + jx[2] * wv[2][j];
        ty3[j] = jy[0] * wv[0][j] + jy[1] * wv[1][j] + jy[2] * wv[2][j];
    }
    for (int j = 0; j < 3; ++j) {
        ax[j] = tx3[0] * m[0][j] + tx3[1] * m[1][j] + tx3[2] * m[2][j];
        ay[j] = ty3[0] * m[0][j] + ty3[1] * m[1][j] + ty3[2] * m[2][j];
    }
    float a = ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2];
    const float b = ax[0] * ay[0] + ax[1] * ay[1] + ax[2] * ay[2];
    float cc = ay[0] * ay[0] + ay[1] * ay[1] + ay[2] * ay[2];

    const float detBefore = a * cc - b * b;
    a = a + 0.3f;
    cc = cc + 0.3f;
    const float det = a * cc - b * b;
    if (!(det > 1e-12f)) return cull();
    float alpha = opacity;
    if (f.antialias != 0) alpha = alpha * std::sqrt(std::fmax(detBefore, 0.0f) / det);
    if (!(alpha >= 1.0f / 255.0f)) return cull();
    const F3 conic{cc / det, -b / det, a / det};
    const float cutoff = cutoffPower(alpha);
    // footprintExtent, frame.slang:142-146
    const float det2 = conic.x * conic.z - conic.y * conic.y;
    const float inv = det2 > 1e-20f ? 1.0f / det2 : 0.0f;
    const float ex = std::sqrt(std::fmax(cutoff * conic.z * inv, 0.0f));
    const float ey = std::sqrt(std::fmax(cutoff * conic.x * inv, 0.0f));
    const Rect rect = tileRect(f, cx, cy, ex, ey);
    if (rect.x0 > rect.x1 || rect.y0 > rect.y1) return cull();

    uint32_t touched = 0;
    for (uint32_t ty = rect.y0; ty <= rect.y1; ++ty)
        for (uint32_t tx = rect.x0; tx <= rect.x1; ++tx)
            if (tileTouched(f, cx, cy, conic, cutoff, tx, ty)) touched += 1;
    if (touched == 0) return cull();

    const F3 base = src.base(i);
    const uint32_t degree = std::min(degreeOf(src.restPerColour()), f.shLimit);
    const F3 dir = normalize3(F3{p.x - f.eye[0], p.y - f.eye[1], p.z - f.eye[2]});
    const F3 rest = evaluateRest(src.shRow(i), degree, dir, src.restOffset());
    F3 colour{std::fmax(base.x + rest.x, 0.0f), std::fmax(base.y + rest.y, 0.0f),
              std::fmax(base.z + rest.z, 0.0f)};
    if (fate.graded) colour = editGrade(f.edit, colour);

    Record rec;
    rec.screen[0] = cx; rec.screen[1] = cy; rec.screen[2] = t.z; rec.screen[3] = cutoff;
    rec.conic[0] = conic.x; rec.conic[1] = conic.y; rec.conic[2] = conic.z; rec.conic[3] = alpha;
    rec.colour[0] = colour.x; rec.colour[1] = colour.y; rec.colour[2] = colour.z; rec.colour[3] = 0.0f;
    out.proj[slot] = rec;
    out.rects[slot] = rect;
    out.touched[slot] = touched;
    out.visible[slot] = 1;
    out.keys[slot] = fbits(t.z) >> 7;
}

// A point instance's object-to-view rows (TileRasterizer.cpp:357-358); points
// take no edit and need no eye.
void setPointObject(Frame& f, const lrt_projection& pr, const lrt_point_instance& inst) {
    const M4 objectToView = mul4(toM4(pr.world_to_view), toM4(inst.object_to_world));
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) f.m[r * 4 + c] = static_cast<float>(objectToView.at(r, c));
    f.edit = lrt_splat_edit{};
}

// shaders/lrt/splat/points_project.slang:35-86, with pointRadius from
// shaders/lrt/points/point_frame.slang:38-44: an opaque disc of the point's
// radius in pixels (never below half a pixel), cut at one radius, alpha one,
// colour.w one. A culled point's record is zeros (the reference leaves it
// unwritten; nothing reads it).
void projectPoint(const Frame& f, const lrt_gpu_points& c, const lrt_point_style& st, uint32_t i, Projected& out) {
    const uint32_t slot = f.base + i;
    auto cull = [&] {
        out.touched[slot] = 0;
        out.visible[slot] = 0;
        out.keys[slot] = 0x00FFFFFFu;
        out.rects[slot] = {1, 1, 0, 0};
        out.proj[slot] = Record{};
    };
    const float* pos = static_cast<const float*>(c.positions) + size_t{i} * 4;
    const F3 t = toView(f, F3{pos[0], pos[1], pos[2]});
    if (!(t.z > f.nearZ) || t.z > f.farZ) return cull();
    float radius = st.size_mode == 1 ? st.size * 0.5f
                                     : (f.ortho != 0 ? st.size * 0.5f * f.focalX : st.size * 0.5f * f.focalX / t.z);
    radius = std::fmax(radius, 0.5f);
    const float invZ = f.ortho != 0 ? 1.0f : 1.0f / t.z;
    const float cx = f.focalX * t.x * invZ + f.centreX;
    const float cy = f.focalY * t.y * invZ + f.centreY;
    const F3 conic{1.0f / (radius * radius), 0.0f, 1.0f / (radius * radius)};
    const float cutoff = 1.0f;
    const Rect rect = tileRect(f, cx, cy, radius, radius);
    if (rect.x0 > rect.x1 || rect.y0 > rect.y1) return cull();
    uint32_t touched = 0;
    for (uint32_t ty = rect.y0; ty <= rect.y1; ++ty)
        for (uint32_t tx = rect.x0; tx <= rect.x1; ++tx)
            if (tileTouched(f, cx, cy, conic, cutoff, tx, ty)) touched += 1;
    if (touched == 0) return cull();
    float rgb[3] = {st.colour[0], st.colour[1], st.colour[2]};
    if (st.constant_colour == 0) {
        const uint32_t* col = static_cast<const uint32_t*>(c.colours) + size_t{i} * 2;
        rgb[0] = lowHalf(col[0]);
        rgb[1] = highHalf(col[0]);
        rgb[2] = lowHalf(col[1]);
    }
    Record rec;
    rec.screen[0] = cx; rec.screen[1] = cy; rec.screen[2] = t.z; rec.screen[3] = cutoff;
    rec.conic[0] = conic.x; rec.conic[1] = conic.y; rec.conic[2] = conic.z; rec.conic[3] = 1.0f;
    rec.colour[0] = rgb[0]; rec.colour[1] = rgb[1]; rec.colour[2] = rgb[2]; rec.colour[3] = 1.0f;
    out.proj[slot] = rec;
    out.rects[slot] = rect;
    out.touched[slot] = touched;
    out.visible[slot] = 1;
    out.keys[slot] = fbits(t.z) >> 7;
}

// What a composite frame has under its splats (splat_blend.slang:11-16):
// the layer's linear premultiplied colour and view depth, or nothing.
struct Under {
    const float* colour = nullptr;   // width*height float4
    const float* depth = nullptr;    // width*height
};

// shaders/lrt/splat/splat_blend.slang:23-108. `composite` is the
// splatBlendComposite entry (:116-120): discs (colour.w > 0.5) end the walk as
// an opaque hit, and so does the under layer (a pair at or behind its depth).
void blendPixel(const Frame& f, const std::vector<Record>& proj, const uint32_t* pairSlots,
                const uint32_t* ranges, uint32_t px, uint32_t py, float* colour, float* depth,
                std::vector<uint32_t>* contributors = nullptr, bool composite = false,
                const Under* under = nullptr) {
    const uint32_t tile = (py / kTile) * f.tilesX + px / kTile;
    const uint32_t start = ranges[tile * 2];
    const uint32_t end = ranges[tile * 2 + 1];
    const float pxf = static_cast<float>(px) + 0.5f;
    const float pyf = static_cast<float>(py) + 0.5f;
    const uint64_t at = uint64_t{py} * f.width + px;
    const bool hasUnder = composite && under != nullptr && under->colour != nullptr;
    const float underZ = hasUnder ? under->depth[at] : 0.0f;
    const bool underHit = hasUnder && underZ > 0.0f;
    float rgb[3] = {0.0f, 0.0f, 0.0f};
    float T = 1.0f;
    float depthSum = 0.0f;
    float depthAt = -1.0f;
    bool opaqueHit = false;
    float opaque[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    float opaqueZ = 0.0f;
    for (uint32_t k = start; k < end; ++k) {
        const Record& rec = proj[pairSlots[k]];
        if (underHit && rec.screen[2] >= underZ) break;
        const float dx = pxf - rec.screen[0];
        const float dy = pyf - rec.screen[1];
        // splat_blend.slang:58, its two sums fused as a GPU compiler contracts them.
        const float t = rec.conic[0] * dx * dx;
        const float u = std::fma(2.0f * rec.conic[1] * dx, dy, t);
        const float power = std::fma(rec.conic[2] * dy, dy, u);
        if (power > rec.screen[3]) continue;
        if (composite && rec.colour[3] > 0.5f) {
            opaqueHit = true;
            opaque[0] = rec.colour[0];
            opaque[1] = rec.colour[1];
            opaque[2] = rec.colour[2];
            opaque[3] = 1.0f;
            opaqueZ = rec.screen[2];
            break;
        }
        const float alpha = std::fmin(0.99f, rec.conic[3] * expImpl(-0.5f * power));
        if (alpha < 1.0f / 255.0f) continue;
        const float weight = T * alpha;
        rgb[0] = std::fma(weight, rec.colour[0], rgb[0]);   // splat_blend.slang:72-74, fused
        rgb[1] = std::fma(weight, rec.colour[1], rgb[1]);
        rgb[2] = std::fma(weight, rec.colour[2], rgb[2]);
        depthSum = std::fma(weight, rec.screen[2], depthSum);
        T = T * (1.0f - alpha);
        if (depthAt < 0.0f && 1.0f - T >= f.depthThreshold) depthAt = rec.screen[2];
        if (contributors != nullptr) contributors->push_back(pairSlots[k]);
        if (T < 1e-4f) break;
    }
    if (!opaqueHit && underHit) {
        opaqueHit = true;
        for (int c = 0; c < 4; ++c) opaque[c] = under->colour[at * 4 + c];
        opaqueZ = underZ;
    }
    const float coverage = 1.0f - T;
    float lin[3] = {rgb[0], rgb[1], rgb[2]};
    if (f.linearise != 0 && coverage > 1e-6f) {
        for (int k = 0; k < 3; ++k) lin[k] = srgbToLinear(rgb[k] / coverage) * coverage;
    }
    float behind[4] = {f.bg[0], f.bg[1], f.bg[2], f.bg[3]};
    if (opaqueHit) {
        for (int c = 0; c < 4; ++c) behind[c] = opaque[c];
        depthSum = depthSum + T * opaqueZ;
        if (depthAt < 0.0f) depthAt = opaqueZ;
    }
    colour[at * 4 + 0] = lin[0] + T * behind[0];
    colour[at * 4 + 1] = lin[1] + T * behind[1];
    colour[at * 4 + 2] = lin[2] + T * behind[2];
    colour[at * 4 + 3] = coverage + T * behind[3];
    const float total = opaqueHit ? 1.0f : coverage;
    depth[at] = f.depthMode == 0 ? (total > 1e-6f ? depthSum / total : 0.0f) : std::fmax(depthAt, 0.0f);
}

uint64_t totalSplats(const lrt_splat_instance* inst, uint32_t n) {
    uint64_t total = 0;
    for (uint32_t k = 0; k < n; ++k)
        if (inst[k].splats != nullptr) total += inst[k].splats->count;
    return total;
}

}   // namespace

extern "C" {

uint32_t ora_abi_version(void) { return LRT_ABI_VERSION; }
float ora_exp(float x) { return expImpl(x); }
float ora_log(float x) { return logImpl(x); }
float ora_pow(float x, float y) { return powImpl(x, y); }
uint16_t ora_f32_to_f16(float f) { return static_cast<uint16_t>(floatToHalf(f)); }
float ora_f16_to_f32(uint16_t h) { return halfToFloat(h); }

void ora_math_eval(int fn, const float* x, float* y, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) {
        switch (fn) {
            case 0: y[i] = expImpl(x[i]); break;
            case 6: y[i] = expImpl(x[i]); break;   // the device's in-range form, -87 <= x <= 88
            case 1: y[i] = logImpl(x[i]); break;
            case 2: y[i] = srgbToLinear(x[i]); break;
            case 3: y[i] = cutoffPower(x[i]); break;
            case 4: {
                const uint32_t h = floatToHalf(x[i]);
                std::memcpy(&y[i], &h, 4);
                break;
            }
            case 5: {
                const uint32_t h = packHalves(x[i], -0.5f * x[i]);
                std::memcpy(&y[i], &h, 4);
                break;
            }
            default: y[i] = NAN; break;
        }
    }
}

int ora_camera_looking_at(const double eye[3], const double target[3], const double up[3],
                          lrt_camera* out) {
    // Camera.cpp:9-13 -> Transform.h lookAt with the -Z look axis.
    std::memset(out, 0, sizeof(*out));
    const M4 id = M4::identity();
    std::memcpy(out->camera_to_world, id.m, sizeof(id.m));
    // Lens defaults, Camera.h:23-44
    out->lens.orthographic = 0;
    out->lens.focal = 50.0;
    out->lens.haperture = 24.576;
    out->lens.vaperture = 18.672;
    out->lens.near_z = 0.1;
    out->lens.far_z = 10000.0;
    out->lens.window_scale[0] = out->lens.window_scale[1] = 1.0;
    const D3 e{eye[0], eye[1], eye[2]};
    const D3 f = normalisedd(sub(D3{target[0], target[1], target[2]}, e));
    M4 o = M4::identity();
    if (lengthd(f) < 1e-12) {
        o.at(0, 3) = e.x;
        o.at(1, 3) = e.y;
        o.at(2, 3) = e.z;
    } else {
        const D3 zAxis = scale(f, -1.0);
        D3 xAxis = normalisedd(crossd(D3{up[0], up[1], up[2]}, zAxis));
        if (lengthd(xAxis) < 1e-12) {
            xAxis = normalisedd(crossd(D3{0.0, 0.0, 1.0}, zAxis));
            if (lengthd(xAxis) < 1e-12) xAxis = {1.0, 0.0, 0.0};
        }
        const D3 yAxis = crossd(zAxis, xAxis);
        o.at(0, 0) = xAxis.x; o.at(0, 1) = yAxis.x; o.at(0, 2) = zAxis.x; o.at(0, 3) = e.x;
        o.at(1, 0) = xAxis.y; o.at(1, 1) = yAxis.y; o.at(1, 2) = zAxis.y; o.at(1, 3) = e.y;
        o.at(2, 0) = xAxis.z; o.at(2, 1) = yAxis.z; o.at(2, 2) = zAxis.z; o.at(2, 3) = e.z;
    }
    std::memcpy(out->camera_to_world, o.m, sizeof(o.m));
    return LRT_OK;
}

int ora_projection_for(const lrt_camera* camera, uint32_t width, uint32_t height,
                       lrt_projection* out) {
    // Camera.cpp:15-48
    std::memset(out, 0, sizeof(*out));
    const M4 c2w = toM4(camera->camera_to_world);
    M4 flip = M4::identity();
    flip.at(2, 2) = -1.0;
    M4 view = mul4(flip, inverseAffine(c2w));
    if (std::fabs(camera->lens.window_roll) > 1e-12) {
        const double rad = camera->lens.window_roll * (3.14159265358979323846 / 180.0);
        const double c = std::cos(rad);
        const double s = std::sin(rad);
        M4 rz = M4::identity();
        rz.at(0, 0) = c; rz.at(0, 1) = -s;
        rz.at(1, 0) = s; rz.at(1, 1) = c;
        view = mul4(rz, view);
    }
    std::memcpy(out->world_to_view, view.m, sizeof(view.m));
    const double w = static_cast<double>(width);
    const double h = static_cast<double>(height);
    const double focal = w * std::max(camera->lens.focal, 1e-9) / std::max(camera->lens.haperture, 1e-9);
    out->focal_x = focal * camera->lens.window_scale[0];
    out->focal_y = focal * camera->lens.window_scale[1];
    out->centre_x = w * 0.5 + camera->lens.window_translate[0] * w * 0.5;
    out->centre_y = h * 0.5 + camera->lens.window_translate[1] * w * 0.5;
    out->near_z = camera->lens.near_z;
    out->far_z = camera->lens.far_z;
    out->orthographic = camera->lens.orthographic ? 1u : 0u;
    out->eye_world[0] = c2w.at(0, 3);
    out->eye_world[1] = c2w.at(1, 3);
    out->eye_world[2] = c2w.at(2, 3);
    return LRT_OK;
}

int ora_pack_splats(const float* raw, uint32_t count, uint32_t fpr, uint32_t filePerColour,
                    uint32_t keep, float* positions, uint32_t* shape, uint32_t* sh,
                    uint32_t* kept) {
    // splat_validate.slang:14-29 + splat_decode.slang:20-91 + splat_encoding.slang:25-69,
    // for the 3DGS PLY encoding (logit opacity, log scale, SH DC, rest colour-outer).
    if (keep > filePerColour || fpr < 14 + 3 * filePerColour) return LRT_INVALID_ARGUMENT;
    const uint32_t shWords = std::max<uint32_t>((keep * 3 + 1) / 2, 1);
    uint32_t j = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const float* r = raw + size_t{i} * fpr;
        const float a = 1.0f / (1.0f + expImpl(-r[3]));
        bool finite = true;
        for (int k : {0, 1, 2, 4, 5, 6}) finite = finite && std::isfinite(r[k]);
        for (int k : {4, 5, 6}) finite = finite && std::fabs(r[k]) < 60.0f;
        if (!(finite && a >= 1.0f / 255.0f)) continue;
        float* pos = positions + size_t{j} * 4;
        pos[0] = r[0]; pos[1] = r[1]; pos[2] = r[2]; pos[3] = saturatef(a);
        const float q[4] = {r[8], r[9], r[10], r[7]};   // (x, y, z, w)
        const float ql = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        const float identity[4] = {0.0f, 0.0f, 0.0f, 1.0f};
        uint32_t* s = shape + size_t{j} * 4;
        s[0] = encodeQuaternion(ql > 1e-8f ? q : identity);
        const float b0 = 0.5f + kSH0 * r[11], b1 = 0.5f + kSH0 * r[12], b2 = 0.5f + kSH0 * r[13];
        s[1] = packHalves(halfSafe(r[4]), halfSafe(r[5]));
        s[2] = packHalves(halfSafe(r[6]), halfSafe(b0));
        s[3] = packHalves(halfSafe(b1), halfSafe(b2));
        uint32_t* row = sh + size_t{j} * shWords;
        std::fill(row, row + shWords, 0u);
        uint32_t n = 0;
        for (uint32_t basis = 0; basis < keep; ++basis)
            for (uint32_t colour = 0; colour < 3; ++colour, ++n) {
                const float v = r[14 + colour * filePerColour + basis];
                row[n / 2] |= (floatToHalf(halfSafe(v)) & 0xFFFFu) << ((n & 1u) * 16);
            }
        ++j;
    }
    *kept = j;
    return LRT_OK;
}

}  // extern "C"

namespace {

// The frame after projection: counts, the reference's two sorts, ranges and
// the blend (TileRasterizer.cpp:382-484). `project` fills P. When `crop` is
// given, the slots that contribute to each pixel inside it are recorded in
// blend order (what a gradient check needs to hold the discrete choices of
// the frame fixed).
struct Crop {
    uint32_t x0, y0, w, h;
    std::vector<std::vector<uint32_t>> lists;
};

template <class ProjectFn>
int renderImpl(const lrt_projection* pr, uint64_t total, const lrt_render_settings* s, ora_frame_out* out,
               uint32_t threads, ProjectFn&& project, Crop* crop, bool composite = false,
               const Under* under = nullptr) {
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    if (s->width == 0 || s->height == 0) return LRT_INVALID_ARGUMENT;
    if (total > 0xFFFFFFFFull) return LRT_UNSUPPORTED;
    Frame f = frameFor(*pr, *s);
    const uint32_t tiles = f.tilesX * f.tilesY;
    const uint32_t slots = static_cast<uint32_t>(total);
    Projected P;
    P.proj.assign(slots, Record{});
    P.rects.assign(slots, Rect{1, 1, 0, 0});
    P.touched.assign(slots, 0);
    P.visible.assign(slots, 0);
    P.keys.assign(slots, 0x00FFFFFFu);

    Clock::time_point t = Clock::now();
    project(f, P, threads);
    out->stage_ms[0] = msSince(t);

    // Counts (TileRasterizer.cpp:382-397).
    std::vector<uint32_t> visibleSlots;
    uint64_t pairs = 0;
    for (uint32_t i = 0; i < slots; ++i) {
        if (P.visible[i]) visibleSlots.push_back(i);
        pairs += P.touched[i];
    }
    out->stage_ms[2] = msSince(t);

    // Depth sort of the visible (splat_compact.slang:16-26, then RadixSort on
    // 24 bits, TileRasterizer.cpp:401-412): stable, ties in slot order.
    std::vector<uint32_t> order = visibleSlots;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return P.keys[a] < P.keys[b]; });
    out->stage_ms[1] = msSince(t);

    // Gather counts + prefix + emit (TileRasterizer.cpp:418-438,
    // splat_gather_counts.slang:11-19, splat_emit.slang:17-50).
    std::vector<uint64_t> offsets(order.size() + 1, 0);
    for (size_t k = 0; k < order.size(); ++k) offsets[k + 1] = offsets[k] + P.touched[order[k]];
    std::vector<uint32_t> pairTiles(pairs), pairSlots(pairs);
    parallelFor(order.size(), threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t k = b; k < e; ++k) {
            const uint32_t sl = order[k];
            const Record& rec = P.proj[sl];
            const Rect rc = P.rects[sl];
            const F3 conic{rec.conic[0], rec.conic[1], rec.conic[2]};
            uint64_t w = 0;
            const uint32_t expected = P.touched[sl];
            for (uint32_t ty = rc.y0; ty <= rc.y1 && w < expected; ++ty)
                for (uint32_t tx = rc.x0; tx <= rc.x1 && w < expected; ++tx) {
                    if (!tileTouched(f, rec.screen[0], rec.screen[1], conic, rec.screen[3], tx, ty)) continue;
                    pairTiles[offsets[k] + w] = ty * f.tilesX + tx;
                    pairSlots[offsets[k] + w] = sl;
                    ++w;
                }
        }
    });
    out->stage_ms[3] = msSince(t);

    // Stable sort of the pairs by tile (TileRasterizer.cpp:444-445): a stable
    // counting sort is the same permutation as the reference's LSD radix.
    std::vector<uint64_t> tileStart(tiles + 1, 0);
    for (uint64_t k = 0; k < pairs; ++k) tileStart[pairTiles[k] + 1] += 1;
    for (uint32_t k = 0; k < tiles; ++k) tileStart[k + 1] += tileStart[k];
    std::vector<uint32_t> sortedTiles(pairs), sortedSlots(pairs);
    {
        std::vector<uint64_t> cursor(tileStart.begin(), tileStart.end() - 1);
        for (uint64_t k = 0; k < pairs; ++k) {
            const uint64_t at = cursor[pairTiles[k]]++;
            sortedTiles[at] = pairTiles[k];
            sortedSlots[at] = pairSlots[k];
        }
    }
    // splat_tiles_clear.slang:8-17 + splat_ranges.slang:11-25
    std::vector<uint32_t> ranges(size_t{tiles} * 2, 0);
    for (uint64_t i = 0; i < pairs; ++i) {
        const uint32_t tt = sortedTiles[i];
        if (i == 0 || sortedTiles[i - 1] != tt) ranges[tt * 2] = static_cast<uint32_t>(i);
        if (i + 1 == pairs || sortedTiles[i + 1] != tt) ranges[tt * 2 + 1] = static_cast<uint32_t>(i + 1);
    }
    out->stage_ms[4] = msSince(t);

    // Blend (splat_blend.slang:110-114): per pixel.
    std::vector<float> colourTmp, depthTmp;
    float* colour = out->colour;
    float* depth = out->depth;
    if (colour == nullptr) {
        colourTmp.resize(size_t{f.width} * f.height * 4);
        colour = colourTmp.data();
    }
    if (depth == nullptr) {
        depthTmp.resize(size_t{f.width} * f.height);
        depth = depthTmp.data();
    }
    const uint8_t* blendTiles = out->blend_tiles;
    parallelFor(f.height, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t py = b; py < e; ++py)
            for (uint32_t px = 0; px < f.width; ++px) {
                if (blendTiles != nullptr && blendTiles[(py / kTile) * f.tilesX + px / kTile] == 0) continue;
                std::vector<uint32_t>* list = nullptr;
                if (crop != nullptr && px >= crop->x0 && px < crop->x0 + crop->w && py >= crop->y0 &&
                    py < crop->y0 + crop->h)
                    list = &crop->lists[(py - crop->y0) * crop->w + (px - crop->x0)];
                blendPixel(f, P.proj, sortedSlots.data(), ranges.data(), px, static_cast<uint32_t>(py), colour,
                           depth, list, composite, under);
            }
    });
    out->stage_ms[5] = msSince(t);

    out->pairs = pairs;
    out->visible = static_cast<uint32_t>(visibleSlots.size());
    out->slots = slots;
    if (out->proj) std::memcpy(out->proj, P.proj.data(), P.proj.size() * sizeof(Record));
    if (out->rects) std::memcpy(out->rects, P.rects.data(), P.rects.size() * sizeof(Rect));
    if (out->touched) std::memcpy(out->touched, P.touched.data(), slots * 4ull);
    if (out->depth_keys) std::memcpy(out->depth_keys, P.keys.data(), slots * 4ull);
    if (out->ranges) std::memcpy(out->ranges, ranges.data(), ranges.size() * 4ull);
    if (pairs <= out->pair_capacity) {
        if (out->pair_tiles) std::memcpy(out->pair_tiles, sortedTiles.data(), pairs * 4ull);
        if (out->pair_slots) std::memcpy(out->pair_slots, sortedSlots.data(), pairs * 4ull);
    }
    return LRT_OK;
}

}  // namespace

extern "C" {

// The Mip-Splatting 3D filter's variance per splat (Yu et al., CVPR 2024,
// section 4.1), as lrt_rast_filter3d defines it: the highest sampling rate
// focal_x / z (focal_x for an orthographic camera) over the cameras whose
// near plane the centre is in front of and whose image, widened by 15% a
// side, its projection falls in; variance coefficient / rate^2; unseen
// splats take the lowest seen rate; none seen: 0.
int ora_filter3d(const lrt_gpu_splats* cloud, const lrt_projection* cams, const uint32_t* sizes, uint32_t camCount,
                 float coefficient, float* out) {
    std::vector<Frame> frames(camCount);
    lrt_splat_instance ident{};
    const double id[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    std::memcpy(ident.object_to_world, id, sizeof(id));
    for (uint32_t k = 0; k < camCount; ++k) {
        lrt_render_settings s{};
        s.width = sizes[2 * k];
        s.height = sizes[2 * k + 1];
        if (s.width == 0 || s.height == 0) return LRT_INVALID_ARGUMENT;
        frames[k] = frameFor(cams[k], s);
        setObject(frames[k], cams[k], ident);
    }
    const float* pos = static_cast<const float*>(cloud->positions);
    float lowest = INFINITY;
    for (uint32_t i = 0; i < cloud->count; ++i) {
        const F3 p{pos[4 * i], pos[4 * i + 1], pos[4 * i + 2]};
        float best = 0.0f;
        for (const Frame& f : frames) {
            const F3 t = toView(f, p);
            if (!(t.z > f.nearZ)) continue;
            const float invZ = f.ortho != 0 ? 1.0f : 1.0f / t.z;
            const float sx = f.focalX * t.x * invZ + f.centreX;
            const float sy = f.focalY * t.y * invZ + f.centreY;
            const float w = static_cast<float>(f.width), h = static_cast<float>(f.height);
            if (!(sx >= -0.15f * w && sx <= 1.15f * w && sy >= -0.15f * h && sy <= 1.15f * h)) continue;
            const float r = f.focalX * invZ;
            if (r > best) best = r;
        }
        out[i] = best;
        if (best > 0.0f && best < lowest) lowest = best;
    }
    for (uint32_t i = 0; i < cloud->count; ++i) {
        float r = out[i];
        if (!(r > 0.0f)) {
            if (!(lowest < INFINITY)) {
                out[i] = 0.0f;
                continue;
            }
            r = lowest;
        }
        out[i] = coefficient / (r * r);
    }
    return LRT_OK;
}

int ora_render(const lrt_projection* pr, const lrt_splat_instance* instances, uint32_t n,
               const lrt_render_settings* s, ora_frame_out* out, uint32_t threads) {
    auto project = [&](const Frame& f, Projected& P, uint32_t th) {
        // TileRasterizer.cpp:290-380 -- project, instance by instance.
        uint32_t base = 0;
        for (uint32_t k = 0; k < n; ++k) {
            const lrt_gpu_splats* c = instances[k].splats;
            if (c == nullptr || c->count == 0) continue;
            Frame fi = f;
            setObject(fi, *pr, instances[k]);
            fi.base = base;
            fi.restPerColour = c->rest_per_colour;
            fi.shWords = c->sh_words;
            parallelFor(c->count, th, [&](uint64_t b, uint64_t e) {
                const PackedSrc src{*c};
                for (uint64_t i = b; i < e; ++i) projectOne(fi, src, static_cast<uint32_t>(i), P);
            });
            base += c->count;
        }
    };
    return renderImpl(pr, totalSplats(instances, n), s, out, threads, project, nullptr);
}

int ora_render_composite(const lrt_projection* pr, const lrt_splat_instance* instances, uint32_t n,
                         const lrt_point_instance* points, uint32_t pointCount, const float* underColour,
                         const float* underDepth, const lrt_render_settings* s, ora_frame_out* out,
                         uint32_t threads) {
    // TileRasterizer.cpp:188-484 with its `points` and `under` arguments:
    // splats first, then the point instances in slots after them (:355-377),
    // and the composite blend when either is given (:464-475).
    uint64_t total = totalSplats(instances, n);
    for (uint32_t k = 0; k < pointCount; ++k)
        if (points[k].points != nullptr) total += points[k].points->count;
    auto project = [&](const Frame& f, Projected& P, uint32_t th) {
        uint32_t base = 0;
        for (uint32_t k = 0; k < n; ++k) {
            const lrt_gpu_splats* c = instances[k].splats;
            if (c == nullptr || c->count == 0) continue;
            Frame fi = f;
            setObject(fi, *pr, instances[k]);
            fi.base = base;
            fi.restPerColour = c->rest_per_colour;
            fi.shWords = c->sh_words;
            parallelFor(c->count, th, [&](uint64_t b, uint64_t e) {
                const PackedSrc src{*c};
                for (uint64_t i = b; i < e; ++i) projectOne(fi, src, static_cast<uint32_t>(i), P);
            });
            base += c->count;
        }
        for (uint32_t k = 0; k < pointCount; ++k) {
            const lrt_gpu_points* c = points[k].points;
            if (c == nullptr || c->count == 0) continue;
            Frame fi = f;
            setPointObject(fi, *pr, points[k]);
            fi.base = base;
            parallelFor(c->count, th, [&](uint64_t b, uint64_t e) {
                for (uint64_t i = b; i < e; ++i) projectPoint(fi, *c, points[k].style, static_cast<uint32_t>(i), P);
            });
            base += c->count;
        }
    };
    const Under under{underColour, underDepth};
    const bool composite = underColour != nullptr || pointCount > 0;
    return renderImpl(pr, total, s, out, threads, project, nullptr, composite, &under);
}

int ora_train_render(const lrt_projection* pr, const lrt_train_params* params, const lrt_render_settings* s,
                     ora_frame_out* out, uint32_t threads, uint32_t crop_x0, uint32_t crop_y0, uint32_t crop_w,
                     uint32_t crop_h, uint32_t* list_offsets, uint32_t* list_slots, uint64_t list_capacity,
                     uint64_t* list_total) {
    lrt_splat_instance inst{};
    const double identity[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    std::memcpy(inst.object_to_world, identity, sizeof(identity));
    auto project = [&](const Frame& f, Projected& P, uint32_t th) {
        Frame fi = f;
        setObject(fi, *pr, inst);
        fi.base = 0;
        parallelFor(params->count, th, [&](uint64_t b, uint64_t e) {
            const RawSrc src{*params};
            for (uint64_t i = b; i < e; ++i) projectOne(fi, src, static_cast<uint32_t>(i), P);
        });
    };
    Crop crop{crop_x0, crop_y0, crop_w, crop_h, {}};
    crop.lists.resize(size_t{crop_w} * crop_h);
    const int code = renderImpl(pr, params->count, s, out, threads, project, (crop_w != 0 && crop_h != 0) ? &crop : nullptr);
    if (code != LRT_OK) return code;
    uint64_t at = 0;
    for (size_t k = 0; k < crop.lists.size(); ++k) {
        if (list_offsets) list_offsets[k] = static_cast<uint32_t>(at);
        for (uint32_t sl : crop.lists[k]) {
            if (list_slots && at < list_capacity) list_slots[at] = sl;
            ++at;
        }
    }
    if (list_offsets) list_offsets[crop.lists.size()] = static_cast<uint32_t>(at);
    if (list_total) *list_total = at;
    return LRT_OK;
}

int ora_reference_render(const lrt_projection* pr, const lrt_splat_instance* instances, uint32_t n,
                         const lrt_render_settings* s, float* colour, float* depth,
                         uint32_t* overflow, uint32_t threads) {
    return ora_reference_render_composite(pr, instances, n, nullptr, 0, s, colour, depth, overflow, threads);
}

int ora_reference_render_composite(const lrt_projection* pr, const lrt_splat_instance* instances, uint32_t n,
                                   const lrt_point_instance* points, uint32_t pointCount,
                                   const lrt_render_settings* s, float* colour, float* depth, uint32_t* overflow,
                                   uint32_t threads) {
    // modules/render/src/ReferenceRenderer.cpp:54-160 with
    // shaders/lrt/reference/reference_project.slang:31-105,
    // reference_points_project.slang:19-41 and reference_blend.slang:24-119.
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    if (s->width == 0 || s->height == 0) return LRT_INVALID_ARGUMENT;
    uint64_t total = totalSplats(instances, n);
    for (uint32_t k = 0; k < pointCount; ++k)
        if (points[k].points != nullptr) total += points[k].points->count;
    Frame f = frameFor(*pr, *s);
    std::vector<std::array<float, 4>> refScreen(total, {0.0f, 0.0f, -1.0f, 0.0f});
    std::vector<std::array<float, 4>> refConic(total), refColour(total);
    uint32_t base = 0;
    for (uint32_t k = 0; k < n; ++k) {
        const lrt_gpu_splats* c = instances[k].splats;
        if (c == nullptr || c->count == 0) continue;
        Frame fi = f;
        setObject(fi, *pr, instances[k]);
        parallelFor(c->count, threads, [&](uint64_t b, uint64_t e) {
            for (uint64_t ii = b; ii < e; ++ii) {
                const uint32_t i = static_cast<uint32_t>(ii);
                const uint32_t slot = base + i;
                const float* pos = static_cast<const float*>(c->positions) + size_t{i} * 4;
                const uint32_t* shape = static_cast<const uint32_t*>(c->shape) + size_t{i} * 4;
                F3 p{pos[0], pos[1], pos[2]};
                const F3 sc{expImpl(lowHalf(shape[1])), expImpl(highHalf(shape[1])),
                            expImpl(lowHalf(shape[2]))};
                const Fate fate = editFate(fi.edit, p, pos[3], sc);
                if (fate.removed) continue;
                const float opacity = fate.opacity;
                const F3 v = toView(fi, p);
                if (!(v.z > fi.nearZ) || v.z > fi.farZ) continue;
                float q[4];
                decodeQuaternion(shape[0], q);
                const float x = q[0], y = q[1], z = q[2], w = q[3];
                const float R[3][3] = {
                    {1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y - w * z), 2.0f * (x * z + w * y)},
                    {2.0f * (x * y + w * z), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z - w * x)},
                    {2.0f * (x * z - w * y), 2.0f * (y * z + w * x), 1.0f - 2.0f * (x * x + y * y)}};
                const float D[3][3] = {{sc.x, 0, 0}, {0, sc.y, 0}, {0, 0, sc.z}};
                auto mm = [](const float A[3][3], const float B[3][3], float C[3][3]) {
                    for (int r = 0; r < 3; ++r)
                        for (int cc = 0; cc < 3; ++cc)
                            C[r][cc] = A[r][0] * B[0][cc] + A[r][1] * B[1][cc] + A[r][2] * B[2][cc];
                };
                auto tr = [](const float A[3][3], float B[3][3]) {
                    for (int r = 0; r < 3; ++r)
                        for (int cc = 0; cc < 3; ++cc) B[r][cc] = A[cc][r];
                };
                float rs[3][3], rsT[3][3], cov3[3][3], W[3][3], WT[3][3], tmp[3][3], covView[3][3];
                mm(R, D, rs);
                tr(rs, rsT);
                mm(rs, rsT, cov3);
                const float Wv[3][3] = {{fi.m[0], fi.m[1], fi.m[2]}, {fi.m[4], fi.m[5], fi.m[6]},
                                        {fi.m[8], fi.m[9], fi.m[10]}};
                for (int r = 0; r < 3; ++r)
                    for (int cc = 0; cc < 3; ++cc) W[r][cc] = Wv[r][cc];
                tr(W, WT);
                mm(cov3, WT, tmp);
                mm(W, tmp, covView);
                float cx, cy;
                float J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                if (fi.ortho) {
                    cx = fi.focalX * v.x + fi.centreX;
                    cy = fi.focalY * v.y + fi.centreY;
                    J[0][0] = fi.focalX;
                    J[1][1] = fi.focalY;
                } else {
                    cx = fi.focalX * v.x / v.z + fi.centreX;
                    cy = fi.focalY * v.y / v.z + fi.centreY;
                    const float lox = (-0.15f * static_cast<float>(fi.width) - fi.centreX) / fi.focalX;
                    const float hix = (1.15f * static_cast<float>(fi.width) - fi.centreX) / fi.focalX;
                    const float loy = (-0.15f * static_cast<float>(fi.height) - fi.centreY) / fi.focalY;
                    const float hiy = (1.15f * static_cast<float>(fi.height) - fi.centreY) / fi.focalY;
                    const float ccx = clampf(v.x / v.z, lox, hix) * v.z;
                    const float ccy = clampf(v.y / v.z, loy, hiy) * v.z;
                    J[0][0] = fi.focalX / v.z;
                    J[0][2] = -fi.focalX * ccx / (v.z * v.z);
                    J[1][1] = fi.focalY / v.z;
                    J[1][2] = -fi.focalY * ccy / (v.z * v.z);
                }
                float JT[3][3], tmp2[3][3], cov2[3][3];
                tr(J, JT);
                mm(covView, JT, tmp2);
                mm(J, tmp2, cov2);
                const float before = cov2[0][0] * cov2[1][1] - cov2[0][1] * cov2[0][1];
                const float a = cov2[0][0] + 0.3f;
                const float b = cov2[0][1];
                const float cc = cov2[1][1] + 0.3f;
                const float det = a * cc - b * b;
                if (!(det > 1e-12f)) continue;
                float alpha = opacity;
                if (fi.antialias != 0) alpha = alpha * std::sqrt(std::fmax(before, 0.0f) / det);
                if (!(alpha >= 1.0f / 255.0f)) continue;
                const F3 baseC{highHalf(shape[2]), lowHalf(shape[3]), highHalf(shape[3])};
                const uint32_t degree = std::min(degreeOf(c->rest_per_colour), fi.shLimit);
                const F3 dir = normalize3(F3{p.x - fi.eye[0], p.y - fi.eye[1], p.z - fi.eye[2]});
                const uint32_t* shRow = static_cast<const uint32_t*>(c->sh) + size_t{i} * c->sh_words;
                const F3 rest = evaluateRest(shRow, degree, dir);
                F3 col{std::fmax(baseC.x + rest.x, 0.0f), std::fmax(baseC.y + rest.y, 0.0f),
                       std::fmax(baseC.z + rest.z, 0.0f)};
                if (fate.graded) col = editGrade(fi.edit, col);
                refScreen[slot] = {cx, cy, v.z, cutoffPower(alpha)};
                refConic[slot] = {cc / det, -b / det, a / det, alpha};
                refColour[slot] = {col.x, col.y, col.z, 0.0f};
            }
        });
        base += c->count;
    }
    for (uint32_t k = 0; k < pointCount; ++k) {
        const lrt_gpu_points* c = points[k].points;
        if (c == nullptr || c->count == 0) continue;
        Frame fi = f;
        setPointObject(fi, *pr, points[k]);
        const lrt_point_style& st = points[k].style;
        parallelFor(c->count, threads, [&](uint64_t b, uint64_t e) {
            for (uint64_t ii = b; ii < e; ++ii) {
                const uint32_t i = static_cast<uint32_t>(ii);
                const uint32_t slot = base + i;
                const float* pos = static_cast<const float*>(c->positions) + size_t{i} * 4;
                const F3 v = toView(fi, F3{pos[0], pos[1], pos[2]});
                if (!(v.z > fi.nearZ) || v.z > fi.farZ) continue;
                const float r = st.size_mode == 1
                                    ? std::fmax(st.size * 0.5f, 0.5f)
                                    : std::fmax(fi.ortho != 0 ? st.size * 0.5f * fi.focalX
                                                              : st.size * 0.5f * fi.focalX / v.z,
                                                0.5f);
                const float cx = fi.ortho != 0 ? fi.focalX * v.x + fi.centreX : fi.focalX * v.x / v.z + fi.centreX;
                const float cy = fi.ortho != 0 ? fi.focalY * v.y + fi.centreY : fi.focalY * v.y / v.z + fi.centreY;
                float rgb[3] = {st.colour[0], st.colour[1], st.colour[2]};
                if (st.constant_colour == 0) {
                    const uint32_t* col = static_cast<const uint32_t*>(c->colours) + size_t{i} * 2;
                    rgb[0] = lowHalf(col[0]);
                    rgb[1] = highHalf(col[0]);
                    rgb[2] = lowHalf(col[1]);
                }
                refScreen[slot] = {cx, cy, v.z, 1.0f};
                refConic[slot] = {1.0f / (r * r), 0.0f, 1.0f / (r * r), 1.0f};
                refColour[slot] = {rgb[0], rgb[1], rgb[2], 1.0f};
            }
        });
        base += c->count;
    }

    constexpr uint32_t kMaxHits = 1024;
    std::atomic<uint32_t> over{0};
    parallelFor(f.height, threads, [&](uint64_t b, uint64_t e) {
        std::vector<float> hitDepth(kMaxHits), hitAlpha(kMaxHits);
        std::vector<uint32_t> hitIndex(kMaxHits), hitDisc(kMaxHits);
        for (uint64_t py = b; py < e; ++py) {
            for (uint32_t px = 0; px < f.width; ++px) {
                const float pxf = static_cast<float>(px) + 0.5f;
                const float pyf = static_cast<float>(py) + 0.5f;
                uint32_t hits = 0;
                bool overflowed = false;
                for (uint64_t sI = 0; sI < total; ++sI) {
                    const auto& sc = refScreen[sI];
                    if (sc[2] < 0.0f) continue;
                    const auto& cn = refConic[sI];
                    const float dx = pxf - sc[0];
                    const float dy = pyf - sc[1];
                    const float power = cn[0] * dx * dx + 2.0f * cn[1] * dx * dy + cn[2] * dy * dy;
                    if (power > sc[3]) continue;
                    const bool disc = refColour[sI][3] > 0.5f;
                    const float alpha = disc ? 1.0f : std::fmin(0.99f, cn[3] * expImpl(-0.5f * power));
                    if (alpha < 1.0f / 255.0f) continue;
                    if (hits == kMaxHits) {
                        overflowed = true;
                        continue;
                    }
                    uint32_t at = hits;
                    while (at > 0 && hitDepth[at - 1] > sc[2]) {
                        hitDepth[at] = hitDepth[at - 1];
                        hitIndex[at] = hitIndex[at - 1];
                        hitAlpha[at] = hitAlpha[at - 1];
                        hitDisc[at] = hitDisc[at - 1];
                        --at;
                    }
                    hitDepth[at] = sc[2];
                    hitIndex[at] = static_cast<uint32_t>(sI);
                    hitAlpha[at] = alpha;
                    hitDisc[at] = disc ? 1u : 0u;
                    ++hits;
                }
                float rgb[3] = {0, 0, 0};
                float T = 1.0f, depthSum = 0.0f, depthAt = -1.0f;
                bool discHit = false;
                float discColour[3] = {0, 0, 0};
                float discZ = 0.0f;
                for (uint32_t k = 0; k < hits; ++k) {
                    if (hitDisc[k] != 0) {
                        discHit = true;
                        for (int c = 0; c < 3; ++c) discColour[c] = refColour[hitIndex[k]][c];
                        discZ = hitDepth[k];
                        break;
                    }
                    const float weight = T * hitAlpha[k];
                    const auto& col = refColour[hitIndex[k]];
                    rgb[0] = rgb[0] + weight * col[0];
                    rgb[1] = rgb[1] + weight * col[1];
                    rgb[2] = rgb[2] + weight * col[2];
                    depthSum = depthSum + weight * hitDepth[k];
                    T = T * (1.0f - hitAlpha[k]);
                    if (depthAt < 0.0f && 1.0f - T >= f.depthThreshold) depthAt = hitDepth[k];
                    if (T < 1e-4f) break;
                }
                const float coverage = 1.0f - T;
                float lin[3] = {rgb[0], rgb[1], rgb[2]};
                if (f.linearise != 0 && coverage > 1e-6f)
                    for (int k = 0; k < 3; ++k) lin[k] = srgbToLinear(rgb[k] / coverage) * coverage;
                const uint64_t at = py * f.width + px;
                float behind[4] = {f.bg[0], f.bg[1], f.bg[2], f.bg[3]};
                if (discHit) {
                    behind[0] = discColour[0];
                    behind[1] = discColour[1];
                    behind[2] = discColour[2];
                    behind[3] = 1.0f;
                    depthSum = depthSum + T * discZ;
                    if (depthAt < 0.0f) depthAt = discZ;
                }
                const float total = discHit ? 1.0f : coverage;
                colour[at * 4 + 0] = lin[0] + T * behind[0];
                colour[at * 4 + 1] = lin[1] + T * behind[1];
                colour[at * 4 + 2] = lin[2] + T * behind[2];
                colour[at * 4 + 3] = coverage + T * behind[3];
                depth[at] = f.depthMode == 0 ? (total > 1e-6f ? depthSum / total : 0.0f)
                                             : std::fmax(depthAt, 0.0f);
                if (overflowed) over.fetch_add(1);
            }
        }
    });
    *overflow = over.load();
    return LRT_OK;
}

int ora_compare_images(const float* a, const float* b, uint32_t width, uint32_t height,
                       uint32_t* histogram, uint32_t* p99, uint32_t* maxOut, uint64_t* over2,
                       uint64_t* pixels) {
    // shaders/lrt/reference/image_compare.slang:20-51 + ReferenceRenderer.cpp:248-297
    auto encode = [](float lin) {
        const float c = saturatef(lin);
        return c <= 0.0031308f ? c * 12.92f : 1.055f * powImpl(c, 1.0f / 2.4f) - 0.055f;
    };
    auto code = [&](float lin) { return static_cast<int>(std::round(encode(lin) * 255.0f)); };
    uint32_t hist[256] = {};
    for (uint64_t i = 0; i < uint64_t{width} * height; ++i) {
        const float* pa = a + i * 4;
        const float* pb = b + i * 4;
        int worst = 0;
        for (int c = 0; c < 3; ++c) worst = std::max(worst, std::abs(code(pa[c]) - code(pb[c])));
        worst = std::max(worst, std::abs(static_cast<int>(std::round(saturatef(pa[3]) * 255.0f)) -
                                         static_cast<int>(std::round(saturatef(pb[3]) * 255.0f))));
        hist[worst] += 1;
    }
    uint64_t total = 0, o2 = 0;
    uint32_t mx = 0;
    for (uint32_t k = 0; k < 256; ++k) {
        total += hist[k];
        if (hist[k] > 0) mx = k;
        if (k > 2) o2 += hist[k];
        if (histogram) histogram[k] = hist[k];
    }
    const uint64_t p99At = total - total / 100;
    uint64_t running = 0;
    uint32_t p = 0;
    for (uint32_t k = 0; k < 256; ++k) {
        running += hist[k];
        if (running >= p99At) {
            p = k;
            break;
        }
    }
    *p99 = p;
    *maxOut = mx;
    *over2 = o2;
    *pixels = total;
    return LRT_OK;
}

int ora_compare_hdr(const float* a, const float* b, uint32_t width, uint32_t height, uint32_t* histogram,
                    float* error) {
    // shaders/lrt/reference/image_compare_hdr.slang:20-60 and floatSum
    // (:82-100): bins eight to an octave from 2^-16 (log2 taken through this
    // restatement's log, as the device takes it), and the relative squared
    // error summed per row, then over rows, with compensated addition.
    uint32_t hist[256] = {};
    auto kahan = [](float& sum, float& carry, float term) {
        const float t = sum + term;
        carry += std::fabs(sum) >= std::fabs(term) ? (sum - t) + term : (term - t) + sum;
        sum = t;
    };
    float total = 0.0f, totalCarry = 0.0f;
    for (uint32_t y = 0; y < height; ++y) {
        float sum = 0.0f, carry = 0.0f;
        for (uint32_t x = 0; x < width; ++x) {
            const float* pa = a + (size_t{y} * width + x) * 4;
            const float* pb = b + (size_t{y} * width + x) * 4;
            float worst = 0.0f, squared = 0.0f;
            for (int c = 0; c < 4; ++c) {
                const float d = std::fabs(pa[c] - pb[c]);
                worst = std::fmax(worst, d / std::fmax(std::fabs(pb[c]), 1e-3f));
                squared += d * d / (pb[c] * pb[c] + 1e-2f);
            }
            const uint32_t bin =
                worst <= 0.0f ? 0u
                              : static_cast<uint32_t>(clampf(std::floor((logImpl(worst) / kLn2Hi + 16.0f) * 8.0f) + 1.0f,
                                                             1.0f, 255.0f));
            hist[bin] += 1;
            kahan(sum, carry, squared * 0.25f);
        }
        kahan(total, totalCarry, sum + carry);
    }
    if (histogram) std::memcpy(histogram, hist, sizeof(hist));
    if (error) *error = total + totalCarry;
    return LRT_OK;
}

uint64_t ora_count_different(const uint32_t* a, const uint32_t* b, uint32_t count) {
    uint64_t n = 0;
    for (uint32_t i = 0; i < count; ++i) n += a[i] != b[i] ? 1 : 0;
    return n;
}

int ora_random_cloud(uint32_t count, uint64_t seed, float minSize, float maxSize, float minOpacity,
                     float maxOpacity, float* raw) {
    // tests/render/SplatFixtures.h:16-85 (CloudBuilder::add + Lcg + randomCloud).
    uint64_t state = 0x853c49e6748fea9bULL ^ seed;
    auto next = [&]() {
        state = state * 6364136223846793005ULL + 1442695040888963407ULL;
        return static_cast<float>((state >> 40) & 0xFFFFFF) / 16777216.0F;
    };
    auto range = [&](float lo, float hi) { return lo + (hi - lo) * next(); };
    const auto logit = [](float a) { return std::log(a / (1.0F - a)); };
    const float sh0 = 0.28209479F;
    for (uint32_t i = 0; i < count; ++i) {
        const float size = std::exp(range(std::log(minSize), std::log(maxSize)));
        const float stretch = range(0.05F, 1.0F);
        float rest[9];
        for (float& v : rest) v = range(-0.3F, 0.3F);
        const float x = range(-2.0F, 2.0F);
        const float y = range(-1.5F, 1.5F);
        const float z = range(-2.0F, 2.0F);
        const float opacity = range(minOpacity, maxOpacity);
        const float thin = range(0.1F, 1.0F);
        float turn[4];
        for (float& v : turn) v = range(-1, 1);
        float dc[3];
        for (float& v : dc) v = range(0.0F, 1.2F);
        float* r = raw + size_t{i} * 23;
        const float vals[14] = {x, y, z, logit(opacity), std::log(size), std::log(size * stretch),
                                std::log(size * thin), turn[0], turn[1], turn[2], turn[3],
                                (dc[0] - 0.5F) / sh0, (dc[1] - 0.5F) / sh0, (dc[2] - 0.5F) / sh0};
        for (int k = 0; k < 14; ++k) r[k] = vals[k];
        for (int k = 0; k < 9; ++k) r[14 + k] = rest[k];
    }
    return LRT_OK;
}

int ora_decode_splats(const float* raw, uint32_t count, const lrt_splat_encoding* e, uint32_t keep,
                      float* positions, uint32_t* shape, uint32_t* sh, uint32_t* kept) {
    // CloudLoader::upload for any encoding (GpuClouds.cpp:151-226):
    // shaders/lrt/scene/splat_validate.slang:19-28, compaction in record
    // order, splat_decode.slang:30-90 with splat_encoding.slang:21-126.
    // Every word of a splat's sh row is written (unused halves zero).
    if (e == nullptr || kept == nullptr) return LRT_INVALID_ARGUMENT;
    const uint32_t s = e->floats_per_record;
    const uint32_t shWords = std::max<uint32_t>((keep * 3 + 1) / 2, 1);
    constexpr float kSH0 = 0.28209479177387814f;
    constexpr float kSqrtHalf = 0.70710678f;
    auto field = [&](uint32_t i, uint32_t f) { return raw[size_t{i} * s + f]; };
    auto opacityOf = [&](float v) {
        if (e->opacity_mode == 0) return 1.0f / (1.0f + expImpl(-v));
        if (e->opacity_mode == 2) return v / 255.0f;
        return v;
    };
    auto logScaleOf = [&](float v) {
        if (e->scale_mode == 2) return v / 16.0f - 10.0f;
        return e->scale_mode == 0 ? v : logImpl(std::fmax(v, 1e-30f));
    };
    auto colourOf = [&](float v) {
        switch (e->colour_mode) {
            case 0: return 0.5f + kSH0 * v;
            case 2: return v / 255.0f;
            case 3: return 0.5f + kSH0 * ((v / 255.0f - 0.5f) / 0.15f);
            case 4: {
                const float c = std::fmax(v, 0.0f);   // linearToSrgb, color.slang:21-24
                return c <= 0.0031308f ? c * 12.92f : 1.055f * powImpl(c, 1.0f / 2.4f) - 0.055f;
            }
            default: return v;
        }
    };
    auto unitOf = [](float v, uint32_t mode) { return mode == 1 ? (v - 128.0f) / 128.0f : v; };
    static const float kSigns[15] = {-1, -1, 1, -1, 1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
    uint32_t j = 0;
    for (uint32_t i = 0; i < count; ++i) {
        F3 p{field(i, e->x) * e->position_scale, field(i, e->y) * e->position_scale,
             field(i, e->z) * e->position_scale};
        if (e->flip_yz != 0) p = F3{p.x, -p.y, -p.z};
        const float a = opacityOf(field(i, e->opacity));
        const float ls[3] = {logScaleOf(field(i, e->scale0)), logScaleOf(field(i, e->scale1)),
                             logScaleOf(field(i, e->scale2))};
        bool finite = std::isfinite(p.x) && std::isfinite(p.y) && std::isfinite(p.z);
        for (float v : ls) finite = finite && std::isfinite(v) && std::fabs(v) < 60.0f;
        if (!(finite && a >= 1.0f / 255.0f)) continue;

        float* pos = positions + size_t{j} * 4;
        pos[0] = p.x;
        pos[1] = p.y;
        pos[2] = p.z;
        pos[3] = saturatef(a);
        float q[4];   // x y z w
        if (e->rotation_mode == 2) {
            q[0] = field(i, e->rot_x) / 127.5f - 1.0f;
            q[1] = field(i, e->rot_y) / 127.5f - 1.0f;
            q[2] = field(i, e->rot_z) / 127.5f - 1.0f;
            q[3] = std::sqrt(std::fmax(0.0f, 1.0f - (q[0] * q[0] + q[1] * q[1] + q[2] * q[2])));
        } else if (e->rotation_mode == 3) {
            uint32_t comp = static_cast<uint32_t>(field(i, e->rot_x)) | (static_cast<uint32_t>(field(i, e->rot_y)) << 16);
            const uint32_t largest = comp >> 30;
            q[0] = q[1] = q[2] = q[3] = 0.0f;
            float sum = 0.0f;
            for (int k = 3; k >= 0; --k) {
                if (static_cast<uint32_t>(k) == largest) continue;
                const float magnitude = kSqrtHalf * static_cast<float>(comp & 511u) / 511.0f;
                q[k] = ((comp >> 9) & 1u) != 0 ? -magnitude : magnitude;
                sum = sum + q[k] * q[k];
                comp = comp >> 10;
            }
            q[largest] = std::sqrt(std::fmax(0.0f, 1.0f - sum));
        } else {
            q[0] = unitOf(field(i, e->rot_x), e->rotation_mode);
            q[1] = unitOf(field(i, e->rot_y), e->rotation_mode);
            q[2] = unitOf(field(i, e->rot_z), e->rotation_mode);
            q[3] = unitOf(field(i, e->rot_w), e->rotation_mode);
        }
        if (e->flip_yz != 0) {
            q[1] = -q[1];
            q[2] = -q[2];
        }
        const float qLength = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        const float unit[4] = {0.0f, 0.0f, 0.0f, 1.0f};
        uint32_t* sw = shape + size_t{j} * 4;
        sw[0] = encodeQuaternion(qLength > 1e-8f ? q : unit);
        const float base[3] = {colourOf(field(i, e->dc0)), colourOf(field(i, e->dc1)), colourOf(field(i, e->dc2))};
        sw[1] = packHalves(halfSafe(ls[0]), halfSafe(ls[1]));
        sw[2] = packHalves(halfSafe(ls[2]), halfSafe(base[0]));
        sw[3] = packHalves(halfSafe(base[1]), halfSafe(base[2]));
        uint32_t* row = sh + size_t{j} * shWords;
        std::fill(row, row + shWords, 0u);
        uint32_t n = 0;
        for (uint32_t basis = 0; basis < keep; ++basis)
            for (uint32_t colour = 0; colour < 3; ++colour, ++n) {
                const uint32_t f = e->rest_colour_outer != 0 ? e->rest_base + colour * e->rest_per_colour + basis
                                                             : e->rest_base + basis * 3 + colour;
                float v = unitOf(field(i, f), e->rest_mode);
                if (e->flip_yz != 0) v = v * kSigns[std::min(basis, 14u)];
                row[n / 2] |= (floatToHalf(halfSafe(v)) & 0xFFFFu) << ((n & 1u) * 16);
            }
        ++j;
    }
    *kept = j;
    return LRT_OK;
}

int ora_pack_points(const float* raw, uint32_t count, uint32_t colourKind, float detail, float* positions,
                    uint32_t* colours, uint32_t* kept) {
    // shaders/lrt/scene/points_validate.slang:19-28 (which points stay),
    // points_decode.slang:24-41 (their layout) and the in-order compaction
    // between them (GpuClouds.cpp:369-430); hash01 from
    // shaders/lrt/common/color.slang:30-34.
    auto hash01 = [](uint32_t v) {
        const uint32_t state = v * 747796405u + 2891336453u;
        const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
        return static_cast<float>((word >> 22u) ^ word) / 4294967295.0f;
    };
    if (kept == nullptr || (count > 0 && (raw == nullptr || positions == nullptr || colours == nullptr)))
        return LRT_INVALID_ARGUMENT;
    uint32_t j = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const float* r = raw + size_t{i} * 6;
        const bool finite = std::isfinite(r[0]) && std::isfinite(r[1]) && std::isfinite(r[2]);
        const bool keep = detail >= 1.0f || hash01(i) < detail;
        if (!(finite && keep)) continue;
        positions[size_t{j} * 4 + 0] = r[0];
        positions[size_t{j} * 4 + 1] = r[1];
        positions[size_t{j} * 4 + 2] = r[2];
        positions[size_t{j} * 4 + 3] = 1.0f;
        float rgb[3] = {1.0f, 1.0f, 1.0f};
        if (colourKind == 1) {
            for (int c = 0; c < 3; ++c) rgb[c] = srgbToLinear(r[3 + c] / 255.0f);
        } else if (colourKind == 2) {
            for (int c = 0; c < 3; ++c) rgb[c] = r[3 + c];
        }
        colours[size_t{j} * 2] = floatToHalf(rgb[0]) | (floatToHalf(rgb[1]) << 16);
        colours[size_t{j} * 2 + 1] = floatToHalf(rgb[2]) | (floatToHalf(1.0f) << 16);
        ++j;
    }
    *kept = j;
    return LRT_OK;
}

int ora_random_points(uint32_t count, uint64_t seed, float* raw) {
    // tests/render/test_points.cpp:22-44 (Lcg + randomPoints): x in [-2, 2],
    // y in [-1.5, 1.5], z in [-2, 2], linear rgb in [0, 1].
    uint64_t state = 0x2545F4914F6CDD1DULL ^ seed;
    auto next = [&]() {
        state = state * 6364136223846793005ULL + 1442695040888963407ULL;
        return static_cast<float>((state >> 40) & 0xFFFFFF) / 16777216.0F;
    };
    auto range = [&](float lo, float hi) { return lo + (hi - lo) * next(); };
    for (uint32_t i = 0; i < count; ++i) {
        float* r = raw + size_t{i} * 6;
        r[0] = range(-2.0F, 2.0F);
        r[1] = range(-1.5F, 1.5F);
        r[2] = range(-2.0F, 2.0F);
        r[3] = range(0.0F, 1.0F);
        r[4] = range(0.0F, 1.0F);
        r[5] = range(0.0F, 1.0F);
    }
    return LRT_OK;
}

}   // extern "C"

// =================================================================== LOD ====
// Levels of detail, restated on the host in the reference's own schedule
// (modules/lod/src/Lod.cpp:86-300 and 349-547 over shaders/lrt/lod/*.slang):
// a stable sort by Morton code, then per level a boundary pass, an exclusive
// prefix sum and the groups pass; leaf moments, merges through the finer
// level's per-splat group index, finalize; per frame the per-level
// selections, the finest level's state, the per-splat selection, and the
// gather in part order.
struct ora_lod {
    uint32_t count = 0, rest = 0, shWords = 0, coarsest = 0, finest = 0;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, extent = 0.0f;
    std::vector<float> positions;               // the store, Morton order: 4 per splat
    std::vector<uint32_t> shape, sh, codes;     // 4, shWords, 1 per splat
    std::vector<uint32_t> groups, starts;       // finest level: group per splat, first splat per group
    struct Level {
        uint32_t level = 0;
        std::vector<float> positions;
        std::vector<uint32_t> shape, sh, cells;
    };
    std::vector<Level> levels;                  // coarsest first
};

namespace {

constexpr uint32_t kOraLodLevels = 10;        // lod_common.slang:36
constexpr uint32_t kOraMomentsHead = 13;      // lod_common.slang:38-40

uint32_t levelShiftOf(uint32_t level) { return 3 * (kOraLodLevels - level); }   // lod_common.slang:64-66

// morton.slang:23-28 by one bit at a time: bit b of x, y, z to bits 3b+2,
// 3b+1, 3b of the code.
uint32_t mortonOf(uint32_t qx, uint32_t qy, uint32_t qz) {
    uint32_t code = 0;
    for (uint32_t b = 0; b < 10; ++b) {
        code |= ((qx >> b) & 1u) << (3 * b + 2);
        code |= ((qy >> b) & 1u) << (3 * b + 1);
        code |= ((qz >> b) & 1u) << (3 * b);
    }
    return code;
}

// morton.slang:30-33.
void cellIndexOf(uint32_t cell, uint32_t idx[3]) {
    idx[0] = idx[1] = idx[2] = 0;
    for (uint32_t b = 0; b < 10; ++b) {
        idx[0] |= ((cell >> (3 * b + 2)) & 1u) << b;
        idx[1] |= ((cell >> (3 * b + 1)) & 1u) << b;
        idx[2] |= ((cell >> (3 * b)) & 1u) << b;
    }
}

uint32_t quantiseUnit(float v, float lo, float extent) {   // morton.slang:25
    const float unit = saturatef((v - lo) / extent);
    const uint32_t q = static_cast<uint32_t>(unit * 1024.0f);
    return q < 1023u ? q : 1023u;
}

// lod_leaf_moments.slang:26-64 for one group [first, end).
void leafMomentsOf(const ora_lod& d, uint32_t first, uint32_t end, float* m) {
    const uint32_t stride = kOraMomentsHead + 3 * d.rest;
    for (uint32_t k = 0; k < stride; ++k) m[k] = 0.0f;
    for (uint32_t i = first; i < end; ++i) {
        const float* p = &d.positions[size_t{i} * 4];
        const uint32_t* row = &d.shape[size_t{i} * 4];
        const float s[3] = {expImpl(lowHalf(row[1])), expImpl(highHalf(row[1])), expImpl(lowHalf(row[2]))};
        float q[4];
        decodeQuaternion(row[0], q);
        const float x = q[0], y = q[1], z = q[2], w = q[3];
        const float r[3][3] = {{1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y - w * z), 2.0f * (x * z + w * y)},
                               {2.0f * (x * y + w * z), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z - w * x)},
                               {2.0f * (x * z - w * y), 2.0f * (y * z + w * x), 1.0f - 2.0f * (x * x + y * y)}};
        float ms[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) ms[a][b] = r[a][b] * s[b];
        float cov[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) cov[a][b] = ms[a][0] * ms[b][0] + ms[a][1] * ms[b][1] + ms[a][2] * ms[b][2];
        const float smallest = std::fmin(std::fmin(s[0], s[1]), s[2]);
        const float area = s[0] * s[1] * s[2] / std::fmax(smallest, 1e-20f);
        const float weight = p[3] * area;
        m[0] += weight;
        m[1] += weight * p[0];
        m[2] += weight * p[1];
        m[3] += weight * p[2];
        m[4] += weight * (cov[0][0] + p[0] * p[0]);
        m[5] += weight * (cov[0][1] + p[0] * p[1]);
        m[6] += weight * (cov[0][2] + p[0] * p[2]);
        m[7] += weight * (cov[1][1] + p[1] * p[1]);
        m[8] += weight * (cov[1][2] + p[1] * p[2]);
        m[9] += weight * (cov[2][2] + p[2] * p[2]);
        m[10] += weight * highHalf(row[2]);
        m[11] += weight * lowHalf(row[3]);
        m[12] += weight * highHalf(row[3]);
        const uint32_t* shRow = d.sh.data() + size_t{i} * d.shWords;
        for (uint32_t h = 0; h < d.rest * 3; ++h) m[kOraMomentsHead + h] += weight * halfAt(shRow, h);
    }
}

void mul3(const float a[3][3], const float b[3][3], float o[3][3]) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o[r][c] = a[r][0] * b[0][c] + a[r][1] * b[1][c] + a[r][2] * b[2][c];
}

float signOf(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }

// lod_finalize.slang:16-40.
void jacobiOf(float a[3][3], float v[3][3]) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) v[r][c] = r == c ? 1.0f : 0.0f;
    for (int sweep = 0; sweep < 6; ++sweep) {
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0;
            const int q = pq == 0 ? 1 : 2;
            const float apq = a[p][q];
            if (std::fabs(apq) < 1e-30f) continue;
            const float theta = (a[q][q] - a[p][p]) / (2.0f * apq);
            const float t = signOf(theta + 1e-30f) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0f));
            const float c = 1.0f / std::sqrt(t * t + 1.0f);
            const float s = t * c;
            float j[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
            j[p][p] = c;
            j[q][q] = c;
            j[p][q] = s;
            j[q][p] = -s;
            float jt[3][3], b[3][3], o[3][3];
            for (int r = 0; r < 3; ++r)
                for (int cc = 0; cc < 3; ++cc) jt[r][cc] = j[cc][r];
            mul3(a, j, b);
            mul3(jt, b, a);
            mul3(v, j, o);
            std::memcpy(v, o, sizeof(o));
        }
    }
}

// packing.slang:76-93.
void quaternionOfAxesOf(const float m[3][3], float q[4]) {
    const float trace = m[0][0] + m[1][1] + m[2][2];
    if (trace > 0.0f) {
        const float s = 0.5f / std::sqrt(trace + 1.0f);
        q[0] = (m[2][1] - m[1][2]) * s, q[1] = (m[0][2] - m[2][0]) * s, q[2] = (m[1][0] - m[0][1]) * s, q[3] = 0.25f / s;
    } else if (m[0][0] > m[1][1] && m[0][0] > m[2][2]) {
        const float s = 2.0f * std::sqrt(1.0f + m[0][0] - m[1][1] - m[2][2]);
        q[0] = 0.25f * s, q[1] = (m[1][0] + m[0][1]) / s, q[2] = (m[0][2] + m[2][0]) / s, q[3] = (m[2][1] - m[1][2]) / s;
    } else if (m[1][1] > m[2][2]) {
        const float s = 2.0f * std::sqrt(1.0f - m[0][0] + m[1][1] - m[2][2]);
        q[0] = (m[1][0] + m[0][1]) / s, q[1] = 0.25f * s, q[2] = (m[2][1] + m[1][2]) / s, q[3] = (m[0][2] - m[2][0]) / s;
    } else {
        const float s = 2.0f * std::sqrt(1.0f - m[0][0] - m[1][1] + m[2][2]);
        q[0] = (m[0][2] + m[2][0]) / s, q[1] = (m[2][1] + m[1][2]) / s, q[2] = 0.25f * s, q[3] = (m[1][0] - m[0][1]) / s;
    }
    const float l = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int k = 0; k < 4; ++k) q[k] = q[k] / l;
}

// lod_finalize.slang:42-96: one group's moments to a packed Gaussian.
void finalizeOf(const float* at, uint32_t rest, uint32_t shWords, float* pos, uint32_t* shape, uint32_t* sh) {
    const float weight = std::fmax(at[0], 1e-30f);
    const float mu[3] = {at[1] / weight, at[2] / weight, at[3] / weight};
    float a[3][3] = {{at[4] / weight, at[5] / weight, at[6] / weight},
                     {at[5] / weight, at[7] / weight, at[8] / weight},
                     {at[6] / weight, at[8] / weight, at[9] / weight}};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) a[r][c] = a[r][c] - mu[r] * mu[c];
    float axes[3][3];
    jacobiOf(a, axes);
    const float det = axes[0][0] * (axes[1][1] * axes[2][2] - axes[1][2] * axes[2][1]) -
                      axes[0][1] * (axes[1][0] * axes[2][2] - axes[1][2] * axes[2][0]) +
                      axes[0][2] * (axes[1][0] * axes[2][1] - axes[1][1] * axes[2][0]);
    if (det < 0.0f)
        for (int r = 0; r < 3; ++r) axes[r][2] = -axes[r][2];
    const float s[3] = {std::sqrt(std::fmax(a[0][0], 1e-14f)), std::sqrt(std::fmax(a[1][1], 1e-14f)),
                        std::sqrt(std::fmax(a[2][2], 1e-14f))};
    const float smallest = std::fmin(std::fmin(s[0], s[1]), s[2]);
    const float area = s[0] * s[1] * s[2] / std::fmax(smallest, 1e-20f);
    const float opacity = std::fmin(at[0] / std::fmax(area, 1e-30f), 0.99f);
    const float base[3] = {at[10] / weight, at[11] / weight, at[12] / weight};
    pos[0] = mu[0], pos[1] = mu[1], pos[2] = mu[2], pos[3] = opacity;
    float q[4];
    quaternionOfAxesOf(axes, q);
    shape[0] = encodeQuaternion(q);
    shape[1] = packHalves(halfSafe(logImpl(s[0])), halfSafe(logImpl(s[1])));
    shape[2] = packHalves(halfSafe(logImpl(s[2])), halfSafe(base[0]));
    shape[3] = packHalves(halfSafe(base[1]), halfSafe(base[2]));
    for (uint32_t w = 0; w < shWords; ++w) sh[w] = 0;
    for (uint32_t h = 0; h < rest * 3; ++h) {
        const uint32_t bits = floatToHalf(halfSafe(at[kOraMomentsHead + h] / weight)) & 0xFFFFu;
        sh[h / 2] |= bits << ((h & 1u) * 16);
    }
}

// lod_cut.slang:12-30.
struct OraCut {
    float lo[3], extent, eye[3], pixelsPerUnit, threshold;
    bool ortho;
    float projectedEdge(uint32_t cell, uint32_t level) const {
        const float edge = extent / static_cast<float>(1u << level);
        if (ortho) return edge * pixelsPerUnit;
        uint32_t idx[3];
        cellIndexOf(cell, idx);
        float d[3];
        for (int k = 0; k < 3; ++k) {
            const float l = lo[k] + static_cast<float>(idx[k]) * edge;
            const float nearest = std::fmin(std::fmax(eye[k], l), l + edge);
            d[k] = nearest - eye[k];
        }
        const float distance = std::fmax(std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), 1e-6f);
        return edge * pixelsPerUnit / distance;
    }
    bool small(uint32_t cell, uint32_t level) const { return threshold > 0.0f && projectedEdge(cell, level) <= threshold; }
};

}  // namespace

extern "C" {

int ora_lod_build(const lrt_gpu_splats* cloud, const float* bounds, float maxGroupFraction, uint32_t coarsestLevel,
                  ora_lod** out) {
    if (cloud == nullptr || out == nullptr || cloud->count == 0) return LRT_INVALID_ARGUMENT;
    const uint32_t n = cloud->count;
    auto d = std::make_unique<ora_lod>();
    d->count = n;
    d->rest = cloud->rest_per_colour;
    d->shWords = cloud->sh_words;
    const float* srcPos = static_cast<const float*>(cloud->positions);
    const uint32_t* srcShape = static_cast<const uint32_t*>(cloud->shape);
    const uint32_t* srcSh = static_cast<const uint32_t*>(cloud->sh);
    // CloudLoader::boundsOf (GpuClouds.cpp:93-125), then Lod.cpp:91-97.
    for (int k = 0; k < 3; ++k) {
        if (bounds != nullptr) {
            d->lo[k] = bounds[k], d->hi[k] = bounds[3 + k];
            continue;
        }
        float lo = 3.4e38f, hi = -3.4e38f;
        for (uint32_t i = 0; i < n; ++i) lo = std::fmin(lo, srcPos[size_t{i} * 4 + k]), hi = std::fmax(hi, srcPos[size_t{i} * 4 + k]);
        d->lo[k] = lo, d->hi[k] = hi;
    }
    float extent = 0.0f;
    for (int k = 0; k < 3; ++k) extent = std::max(extent, d->hi[k] - d->lo[k]);
    extent = std::max(extent, 1e-6f);
    extent *= 1.0001f;
    d->extent = extent;
    // Morton order (lod_morton.slang; RadixSort is stable: ties keep index order).
    std::vector<uint32_t> keys(n), order(n);
    const float e = std::fmax(extent, 1e-20f);
    for (uint32_t i = 0; i < n; ++i) {
        const float* p = srcPos + size_t{i} * 4;
        keys[i] = mortonOf(quantiseUnit(p[0], d->lo[0], e), quantiseUnit(p[1], d->lo[1], e), quantiseUnit(p[2], d->lo[2], e));
        order[i] = i;
    }
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
    d->positions.resize(size_t{n} * 4);
    d->shape.resize(size_t{n} * 4);
    d->sh.resize(size_t{n} * d->shWords);
    d->codes.resize(n);
    for (uint32_t k = 0; k < n; ++k) {   // lod_reorder.slang
        const uint32_t i = order[k];
        d->codes[k] = keys[i];
        std::memcpy(&d->positions[size_t{k} * 4], srcPos + size_t{i} * 4, 16);
        std::memcpy(&d->shape[size_t{k} * 4], srcShape + size_t{i} * 4, 16);
        if (d->shWords > 0) std::memcpy(&d->sh[size_t{k} * d->shWords], srcSh + size_t{i} * d->shWords, d->shWords * 4);
    }
    // Every level's groups (Lod.cpp:151-211).
    struct LevelGroups {
        uint32_t groups = 0;
        std::vector<uint32_t> group, starts, cells;
    };
    std::vector<LevelGroups> lv(kOraLodLevels + 1);
    auto groupsOf = [&](uint32_t level) {
        const uint32_t shift = levelShiftOf(level);
        std::vector<uint32_t> boundary(n), before(n);
        for (uint32_t i = 0; i < n; ++i)   // lod_boundaries.slang
            boundary[i] = (i == 0 || (d->codes[i] >> shift) != (d->codes[i - 1] >> shift)) ? 1u : 0u;
        uint32_t total = 0;
        for (uint32_t i = 0; i < n; ++i) before[i] = total, total += boundary[i];
        LevelGroups& g = lv[level];
        g.groups = total;
        g.group.resize(n);
        g.starts.resize(total);
        g.cells.resize(total);
        for (uint32_t i = 0; i < n; ++i) {   // lod_groups.slang
            const uint32_t grp = before[i] + boundary[i] - 1;
            g.group[i] = grp;
            if (boundary[i] != 0) g.starts[grp] = i, g.cells[grp] = d->codes[i] >> shift;
        }
    };
    const uint32_t coarsest = std::clamp<uint32_t>(coarsestLevel, 1, kOraLodLevels);
    uint32_t finest = coarsest;
    for (uint32_t level = coarsest; level <= kOraLodLevels; ++level) {
        groupsOf(level);
        if (static_cast<float>(lv[level].groups) > maxGroupFraction * static_cast<float>(n) && level > coarsest) break;
        finest = level;
    }
    d->coarsest = coarsest;
    d->finest = finest;
    // Moments from the finest level up, a Gaussian per group (Lod.cpp:213-266).
    const uint32_t stride = kOraMomentsHead + 3 * d->rest;
    std::vector<float> fine;
    std::vector<ora_lod::Level> stored;
    for (uint32_t level = finest + 1; level-- > coarsest;) {
        const LevelGroups& g = lv[level];
        std::vector<float> moments(size_t{g.groups} * stride, 0.0f);
        if (level == finest) {
            for (uint32_t grp = 0; grp < g.groups; ++grp) {
                const uint32_t end = grp + 1 < g.groups ? g.starts[grp + 1] : n;
                leafMomentsOf(*d, g.starts[grp], end, &moments[size_t{grp} * stride]);
            }
        } else {   // lod_merge_moments.slang
            const LevelGroups& f = lv[level + 1];
            for (uint32_t grp = 0; grp < g.groups; ++grp) {
                const uint32_t first = f.group[g.starts[grp]];
                const uint32_t end = grp + 1 < g.groups ? f.group[g.starts[grp + 1]] : f.groups;
                for (uint32_t k = 0; k < stride; ++k) {
                    float sum = 0.0f;
                    for (uint32_t h = first; h < end; ++h) sum += fine[size_t{h} * stride + k];
                    moments[size_t{grp} * stride + k] = sum;
                }
            }
        }
        ora_lod::Level out;
        out.level = level;
        out.positions.resize(size_t{g.groups} * 4);
        out.shape.resize(size_t{g.groups} * 4);
        out.sh.resize(size_t{g.groups} * d->shWords);
        out.cells = g.cells;
        for (uint32_t grp = 0; grp < g.groups; ++grp)
            finalizeOf(&moments[size_t{grp} * stride], d->rest, d->shWords, &out.positions[size_t{grp} * 4],
                       &out.shape[size_t{grp} * 4], out.sh.data() + size_t{grp} * d->shWords);
        if (level == finest) d->groups = g.group, d->starts = g.starts;
        stored.push_back(std::move(out));
        fine = std::move(moments);
    }
    std::reverse(stored.begin(), stored.end());
    d->levels = std::move(stored);
    *out = d.release();
    return LRT_OK;
}

void ora_lod_free(ora_lod* d) { delete d; }

int ora_lod_describe(const ora_lod* d, lrt_lod_info* out) {
    if (d == nullptr || out == nullptr) return LRT_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    out->count = d->count;
    out->rest_per_colour = d->rest;
    out->sh_words = d->shWords;
    out->levels = static_cast<uint32_t>(d->levels.size());
    out->coarsest = d->coarsest;
    out->finest = d->finest;
    for (int k = 0; k < 3; ++k) out->bounds_lo[k] = d->lo[k], out->bounds_hi[k] = d->hi[k];
    out->extent = d->extent;
    for (size_t l = 0; l < d->levels.size(); ++l) {
        out->level_groups[l] = static_cast<uint32_t>(d->levels[l].cells.size());
        out->merged += out->level_groups[l];
    }
    return LRT_OK;
}

// which: 0 store positions, 1 store shape, 2 store sh, 3 codes, 4 finest starts,
// 5 merged positions, 6 merged shape, 7 merged sh, 8 cells (all levels, coarsest first).
int ora_lod_copy(const ora_lod* d, int which, void* dst) {
    if (d == nullptr || dst == nullptr) return LRT_INVALID_ARGUMENT;
    auto put = [&](const void* src, size_t bytes) {
        if (bytes > 0) std::memcpy(dst, src, bytes);
        dst = static_cast<char*>(dst) + bytes;
    };
    switch (which) {
        case 0: put(d->positions.data(), d->positions.size() * 4); break;
        case 1: put(d->shape.data(), d->shape.size() * 4); break;
        case 2: put(d->sh.data(), d->sh.size() * 4); break;
        case 3: put(d->codes.data(), d->codes.size() * 4); break;
        case 4: put(d->starts.data(), d->starts.size() * 4); break;
        case 5: for (const auto& l : d->levels) put(l.positions.data(), l.positions.size() * 4); break;
        case 6: for (const auto& l : d->levels) put(l.shape.data(), l.shape.size() * 4); break;
        case 7: for (const auto& l : d->levels) put(l.sh.data(), l.sh.size() * 4); break;
        case 8: for (const auto& l : d->levels) put(l.cells.data(), l.cells.size() * 4); break;
        default: return LRT_INVALID_ARGUMENT;
    }
    return LRT_OK;
}

// CutSelector::select for one instance, every chunk resident: the drawn cloud
// (capacity: the cloud's splat count) and its counts.
int ora_lod_cut(const ora_lod* d, const lrt_projection* pr, const double objectToWorld[16], float threshold,
                float* positions, uint32_t* shape, uint32_t* sh, uint32_t* splats, uint32_t* merged) {
    if (d == nullptr || pr == nullptr || objectToWorld == nullptr) return LRT_INVALID_ARGUMENT;
    OraCut c{};
    for (int k = 0; k < 3; ++k) c.lo[k] = d->lo[k];
    c.extent = d->extent;
    const M4 toWorld = toM4(objectToWorld);   // Lod.cpp:400-408
    const D3 eye = pointOf(inverseAffine(toWorld), D3{pr->eye_world[0], pr->eye_world[1], pr->eye_world[2]});
    c.eye[0] = static_cast<float>(eye.x), c.eye[1] = static_cast<float>(eye.y), c.eye[2] = static_cast<float>(eye.z);
    double scale = 0.0;
    for (int col = 0; col < 3; ++col)
        scale = std::max(scale, lengthd(D3{toWorld.at(0, col), toWorld.at(1, col), toWorld.at(2, col)}));
    c.pixelsPerUnit = static_cast<float>(pr->orthographic ? pr->focal_x * scale : pr->focal_x);
    c.threshold = threshold;
    c.ortho = pr->orthographic != 0;
    const size_t parts = d->levels.size();
    std::vector<std::vector<uint32_t>> selected(parts + 1);
    std::vector<uint32_t> state;
    for (size_t part = 0; part < parts; ++part) {   // lodCutGroups, lodCutFinest
        const ora_lod::Level& l = d->levels[part];
        selected[part].resize(l.cells.size());
        const bool finest = part + 1 == parts;
        if (finest) state.resize(l.cells.size());
        for (size_t g = 0; g < l.cells.size(); ++g) {
            const bool here = c.small(l.cells[g], l.level);
            const bool above = part != 0 && c.small(l.cells[g] >> 3, l.level - 1);
            selected[part][g] = (here && !above) ? 1u : 0u;
            if (finest) state[g] = (here ? 0u : 1u) | (!here ? 2u : 0u);
        }
    }
    selected[parts].resize(d->count);   // lodCutSplats
    for (uint32_t i = 0; i < d->count; ++i) selected[parts][i] = (state[d->groups[i]] & 2u) != 0 ? 1u : 0u;
    uint32_t drawn = 0, drawnMerged = 0;
    for (size_t part = 0; part <= parts; ++part) {   // prefix sums and lodGather, in part order
        const bool isMerged = part < parts;
        const float* srcPos = isMerged ? d->levels[part].positions.data() : d->positions.data();
        const uint32_t* srcShape = isMerged ? d->levels[part].shape.data() : d->shape.data();
        const uint32_t* srcSh = isMerged ? d->levels[part].sh.data() : d->sh.data();
        for (size_t i = 0; i < selected[part].size(); ++i) {
            if (selected[part][i] == 0) continue;
            if (drawn < d->count) {
                if (positions) std::memcpy(positions + size_t{drawn} * 4, srcPos + i * 4, 16);
                if (shape) std::memcpy(shape + size_t{drawn} * 4, srcShape + i * 4, 16);
                if (sh && d->shWords > 0) std::memcpy(sh + size_t{drawn} * d->shWords, srcSh + i * d->shWords, d->shWords * 4);
            }
            ++drawn;
            if (isMerged) ++drawnMerged;
        }
    }
    if (splats) *splats = drawn - drawnMerged;
    if (merged) *merged = drawnMerged;
    return drawn <= d->count ? LRT_OK : LRT_INTERNAL_ERROR;
}

}  // extern "C"
