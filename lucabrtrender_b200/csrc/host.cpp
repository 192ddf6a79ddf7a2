// Host-side parts of the C-ABI: the camera (Camera::lookingAt and
// projectionFor) and the packing of raw 3DGS records into the GpuSplats
// layout the rasteriser reads.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/lrt_raster.h"
#include "lrt_math.cuh"

namespace {

struct Vec3 {
    double x, y, z;
};
Vec3 sub(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
Vec3 scaled(Vec3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
Vec3 cross(Vec3 a, Vec3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double length(Vec3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
Vec3 normalised(Vec3 a) {
    const double l = length(a);
    return l > 1e-12 ? scaled(a, 1.0 / l) : Vec3{0.0, 0.0, 0.0};
}

void identity(double* m) {
    std::fill(m, m + 16, 0.0);
    m[0] = m[5] = m[10] = m[15] = 1.0;
}

void multiply(const double* a, const double* b, double* out) {
    double o[16];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += a[r * 4 + k] * b[k * 4 + c];
            o[r * 4 + c] = s;
        }
    std::memcpy(out, o, sizeof(o));
}

// Inverse of an affine matrix by cofactors (aofx::xform::inverseAffine).
void inverse_affine(const double* m, double* out) {
    auto at = [&](int r, int c) { return m[r * 4 + c]; };
    const double a00 = at(0, 0), a01 = at(0, 1), a02 = at(0, 2);
    const double a10 = at(1, 0), a11 = at(1, 1), a12 = at(1, 2);
    const double a20 = at(2, 0), a21 = at(2, 1), a22 = at(2, 2);
    const double c00 = a11 * a22 - a12 * a21;
    const double c01 = a12 * a20 - a10 * a22;
    const double c02 = a10 * a21 - a11 * a20;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    const double inv = std::fabs(det) > 1e-18 ? 1.0 / det : 0.0;
    double o[16];
    identity(o);
    o[0] = c00 * inv;
    o[1] = (a02 * a21 - a01 * a22) * inv;
    o[2] = (a01 * a12 - a02 * a11) * inv;
    o[4] = c01 * inv;
    o[5] = (a00 * a22 - a02 * a20) * inv;
    o[6] = (a02 * a10 - a00 * a12) * inv;
    o[8] = c02 * inv;
    o[9] = (a01 * a20 - a00 * a21) * inv;
    o[10] = (a00 * a11 - a01 * a10) * inv;
    const double tx = at(0, 3), ty = at(1, 3), tz = at(2, 3);
    o[3] = -(o[0] * tx + o[1] * ty + o[2] * tz);
    o[7] = -(o[4] * tx + o[5] * ty + o[6] * tz);
    o[11] = -(o[8] * tx + o[9] * ty + o[10] * tz);
    std::memcpy(out, o, sizeof(o));
}

// Smallest-three quaternion, packing.slang:26-50 (normalise by the length).
uint32_t encode_quaternion(const float q0[4]) {
    const float l = std::sqrt(q0[0] * q0[0] + q0[1] * q0[1] + q0[2] * q0[2] + q0[3] * q0[3]);
    float q[4] = {q0[0] / l, q0[1] / l, q0[2] / l, q0[3] / l};
    uint32_t largest = 0;
    float best = std::fabs(q[0]);
    for (uint32_t k = 1; k < 4; ++k)
        if (std::fabs(q[k]) > best) {
            best = std::fabs(q[k]);
            largest = k;
        }
    if (q[largest] < 0.0f)
        for (float& v : q) v = -v;
    uint32_t word = largest;
    uint32_t shift = 22;
    for (uint32_t k = 0; k < 4; ++k) {
        if (k == largest) continue;
        const float unit = std::fmin(std::fmax(q[k] / 0.70710678f * 0.5f + 0.5f, 0.0f), 1.0f);
        word |= static_cast<uint32_t>(std::round(unit * 1023.0f)) << shift;
        shift -= 10;
    }
    return word;
}

float half_safe(float v) { return std::fmin(std::fmax(v, -65000.0f), 65000.0f); }
uint32_t pack_halves(float a, float b) {
    return (lrt::float_to_half(a) & 0xFFFFu) | ((lrt::float_to_half(b) & 0xFFFFu) << 16);
}

}  // namespace

extern "C" {

int lrt_camera_looking_at(const double eye[3], const double target[3], const double up[3], lrt_camera* out) {
    if (eye == nullptr || target == nullptr || up == nullptr || out == nullptr) return LRT_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    // Lens defaults (modules/render/include/lrt/render/Camera.h:23-44).
    out->lens.focal = 50.0;
    out->lens.haperture = 24.576;
    out->lens.vaperture = 18.672;
    out->lens.near_z = 0.1;
    out->lens.far_z = 10000.0;
    out->lens.window_scale[0] = out->lens.window_scale[1] = 1.0;
    // A camera looks down its own -Z: +Z of its frame points away from the target.
    double* m = out->camera_to_world;
    identity(m);
    const Vec3 e{eye[0], eye[1], eye[2]};
    const Vec3 f = normalised(sub(Vec3{target[0], target[1], target[2]}, e));
    if (length(f) >= 1e-12) {
        const Vec3 zAxis = scaled(f, -1.0);
        Vec3 xAxis = normalised(cross(Vec3{up[0], up[1], up[2]}, zAxis));
        if (length(xAxis) < 1e-12) {
            xAxis = normalised(cross(Vec3{0.0, 0.0, 1.0}, zAxis));
            if (length(xAxis) < 1e-12) xAxis = {1.0, 0.0, 0.0};
        }
        const Vec3 yAxis = cross(zAxis, xAxis);
        m[0] = xAxis.x; m[1] = yAxis.x; m[2] = zAxis.x;
        m[4] = xAxis.y; m[5] = yAxis.y; m[6] = zAxis.y;
        m[8] = xAxis.z; m[9] = yAxis.z; m[10] = zAxis.z;
    }
    m[3] = e.x;
    m[7] = e.y;
    m[11] = e.z;
    return LRT_OK;
}

int lrt_projection_for(const lrt_camera* camera, uint32_t width, uint32_t height, lrt_projection* out) {
    if (camera == nullptr || out == nullptr) return LRT_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    // The view is the camera's inverse with z negated (+z forward), then the
    // film back's roll about the view's own z.
    double flip[16];
    identity(flip);
    flip[10] = -1.0;
    double inv[16];
    inverse_affine(camera->camera_to_world, inv);
    multiply(flip, inv, out->world_to_view);
    if (std::fabs(camera->lens.window_roll) > 1e-12) {
        const double rad = camera->lens.window_roll * (3.14159265358979323846 / 180.0);
        double rz[16];
        identity(rz);
        rz[0] = std::cos(rad);
        rz[1] = -std::sin(rad);
        rz[4] = std::sin(rad);
        rz[5] = std::cos(rad);
        multiply(rz, out->world_to_view, out->world_to_view);
    }
    const double w = static_cast<double>(width);
    const double h = static_cast<double>(height);
    // W * focal / haperture pixels per unit of x/z (per world unit, orthographic).
    const double focal = w * std::max(camera->lens.focal, 1e-9) / std::max(camera->lens.haperture, 1e-9);
    out->focal_x = focal * camera->lens.window_scale[0];
    out->focal_y = focal * camera->lens.window_scale[1];
    out->centre_x = w * 0.5 + camera->lens.window_translate[0] * w * 0.5;
    out->centre_y = h * 0.5 + camera->lens.window_translate[1] * w * 0.5;
    out->near_z = camera->lens.near_z;
    out->far_z = camera->lens.far_z;
    out->orthographic = camera->lens.orthographic ? 1u : 0u;
    out->eye_world[0] = camera->camera_to_world[3];
    out->eye_world[1] = camera->camera_to_world[7];
    out->eye_world[2] = camera->camera_to_world[11];
    return LRT_OK;
}

int lrt_pack_splats(const float* raw, uint32_t count, uint32_t fpr, uint32_t filePerColour, uint32_t keep,
                    float* positions, uint32_t* shape, uint32_t* sh, uint32_t* kept) {
    // Validation (shaders/lrt/scene/splat_validate.slang:14-29), compaction in
    // record order, and packing (splat_decode.slang:20-91 with the PLY
    // encoding of splat_encoding.slang:29-54).
    if (kept == nullptr || (count > 0 && (raw == nullptr || positions == nullptr || shape == nullptr || sh == nullptr)))
        return LRT_INVALID_ARGUMENT;
    if (keep > filePerColour || fpr < 14 + 3 * filePerColour) return LRT_INVALID_ARGUMENT;
    const uint32_t shWords = std::max<uint32_t>((keep * 3 + 1) / 2, 1);
    // Pass 1: validity and destinations (parallel over records).
    std::vector<uint8_t> valid(count);
    const uint32_t threads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    auto parallel = [&](auto&& fn) {
        if (count < 65536 || threads == 1) {
            fn(0u, count);
            return;
        }
        std::vector<std::thread> pool;
        for (uint32_t t = 0; t < threads; ++t) {
            const uint32_t b = static_cast<uint32_t>(uint64_t{count} * t / threads);
            const uint32_t e = static_cast<uint32_t>(uint64_t{count} * (t + 1) / threads);
            pool.emplace_back([&, b, e] { fn(b, e); });
        }
        for (auto& th : pool) th.join();
    };
    parallel([&](uint32_t b, uint32_t e) {
        for (uint32_t i = b; i < e; ++i) {
            const float* r = raw + size_t{i} * fpr;
            const float a = 1.0f / (1.0f + lrt::lrt_exp(-r[3]));
            bool finite = std::isfinite(r[0]) && std::isfinite(r[1]) && std::isfinite(r[2]) && std::isfinite(r[4]) &&
                          std::isfinite(r[5]) && std::isfinite(r[6]);
            finite = finite && std::fabs(r[4]) < 60.0f && std::fabs(r[5]) < 60.0f && std::fabs(r[6]) < 60.0f;
            valid[i] = (finite && a >= 1.0f / 255.0f) ? 1 : 0;
        }
    });
    std::vector<uint32_t> dest(count);
    uint32_t j = 0;
    for (uint32_t i = 0; i < count; ++i) {
        dest[i] = j;
        j += valid[i];
    }
    *kept = j;
    parallel([&](uint32_t b, uint32_t e) {
        for (uint32_t i = b; i < e; ++i) {
            if (!valid[i]) continue;
            const float* r = raw + size_t{i} * fpr;
            const uint32_t d = dest[i];
            const float a = 1.0f / (1.0f + lrt::lrt_exp(-r[3]));
            float* pos = positions + size_t{d} * 4;
            pos[0] = r[0];
            pos[1] = r[1];
            pos[2] = r[2];
            pos[3] = std::fmin(std::fmax(a, 0.0f), 1.0f);
            const float q[4] = {r[8], r[9], r[10], r[7]};   // stored w x y z; packed as x y z w
            const float ql = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
            const float unit[4] = {0.0f, 0.0f, 0.0f, 1.0f};
            uint32_t* s = shape + size_t{d} * 4;
            s[0] = encode_quaternion(ql > 1e-8f ? q : unit);
            constexpr float kSH0 = 0.28209479177387814f;
            const float b0 = 0.5f + kSH0 * r[11], b1 = 0.5f + kSH0 * r[12], b2 = 0.5f + kSH0 * r[13];
            s[1] = pack_halves(half_safe(r[4]), half_safe(r[5]));
            s[2] = pack_halves(half_safe(r[6]), half_safe(b0));
            s[3] = pack_halves(half_safe(b1), half_safe(b2));
            uint32_t* row = sh + size_t{d} * shWords;
            std::fill(row, row + shWords, 0u);
            uint32_t n = 0;
            for (uint32_t basis = 0; basis < keep; ++basis)
                for (uint32_t colour = 0; colour < 3; ++colour, ++n) {
                    const float v = r[14 + colour * filePerColour + basis];
                    row[n / 2] |= (lrt::float_to_half(half_safe(v)) & 0xFFFFu) << ((n & 1u) * 16);
                }
        }
    });
    return LRT_OK;
}

}  // extern "C"

namespace {

// shaders/lrt/common/color.slang:7-10 and :30-34, on the host.
float srgb_to_linear_host(float c) {
    c = std::fmax(c, 0.0f);
    return c <= 0.04045f ? c / 12.92f : lrt::lrt_pow((c + 0.055f) / 1.055f, 2.4f);
}

float index_hash01(uint32_t v) {
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return static_cast<float>((word >> 22u) ^ word) / 4294967295.0f;
}

}  // namespace

extern "C" int lrt_pack_points(const float* raw, uint32_t count, uint32_t colourKind, float detail, float* positions,
                               uint32_t* colours, uint32_t* kept) {
    // The points half of CloudLoader::upload (GpuClouds.cpp:369-430): which
    // points stay (points_validate.slang:19-28: finite, and thinned to
    // `detail` by an index hash), compacted in order, then their layout
    // (points_decode.slang:24-41).
    if (kept == nullptr) return LRT_INVALID_ARGUMENT;
    *kept = 0;
    if (count > 0 && (raw == nullptr || positions == nullptr || colours == nullptr)) return LRT_INVALID_ARGUMENT;
    if (colourKind > 2) return LRT_INVALID_ARGUMENT;
    uint32_t j = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const float* r = raw + static_cast<size_t>(i) * 6;
        if (!(std::isfinite(r[0]) && std::isfinite(r[1]) && std::isfinite(r[2]))) continue;
        if (!(detail >= 1.0f || index_hash01(i) < detail)) continue;
        float* p = positions + static_cast<size_t>(j) * 4;
        p[0] = r[0];
        p[1] = r[1];
        p[2] = r[2];
        p[3] = 1.0f;
        float rgb[3] = {1.0f, 1.0f, 1.0f};
        for (int c = 0; c < 3; ++c) {
            if (colourKind == 1) rgb[c] = srgb_to_linear_host(r[3 + c] / 255.0f);
            if (colourKind == 2) rgb[c] = r[3 + c];
        }
        colours[static_cast<size_t>(j) * 2] = pack_halves(rgb[0], rgb[1]);
        colours[static_cast<size_t>(j) * 2 + 1] = pack_halves(rgb[2], 1.0f);
        ++j;
    }
    *kept = j;
    return LRT_OK;
}

extern "C" int lrt_splat_encoding_ply(uint32_t restPerColour, lrt_splat_encoding* out) {
    // io::SplatEncoding as the PLY reader fills it for a 3DGS file: x y z,
    // logit opacity, three log scales, rotation w x y z, three DC terms, then
    // the rest coefficients all red, then green, then blue.
    if (out == nullptr || !(restPerColour == 0 || restPerColour == 3 || restPerColour == 8 || restPerColour == 15))
        return LRT_INVALID_ARGUMENT;
    *out = lrt_splat_encoding{};
    out->floats_per_record = 14 + 3 * restPerColour;
    out->x = 0;
    out->y = 1;
    out->z = 2;
    out->opacity = 3;
    out->scale0 = 4;
    out->scale1 = 5;
    out->scale2 = 6;
    out->rot_w = 7;
    out->rot_x = 8;
    out->rot_y = 9;
    out->rot_z = 10;
    out->dc0 = 11;
    out->dc1 = 12;
    out->dc2 = 13;
    out->rest_base = 14;
    out->rest_per_colour = restPerColour;
    out->rest_colour_outer = 1;
    out->position_scale = 1.0f;
    return LRT_OK;
}
