// The backward of the projection, per splat (no reference counterpart: the
// reference renders only). A splat's nine per-pair partials -- d/d(centre x,
// y, conic a, b, c, alpha, colour r, g, b), written by the blend backward at
// the pair's emit index -- are contiguous from the splat's first pair index,
// so they are summed in a fixed order (no atomics, deterministic), then carried
// back through the forward of splat_project.slang:72-169 to the
// parameters: means, log-scales, quaternions (w, x, y, z; normalised in the
// forward), opacity logits and the 16 x 3 SH coefficients (fp32 gradients of
// fp16 values). Every forward intermediate is recomputed from the parameters
// with the forward's own expressions.
#include "kernels.cuh"
#include "raster_common.cuh"

namespace lrt {
namespace {

constexpr uint32_t kThreads = 128;
constexpr uint32_t kMaxChunkViews = 16;   // views one splat_backward_views launch takes
constexpr uint32_t kGradStrideFloats = 12;  // floats per pair in the partials buffer
constexpr float kC1 = 0.4886025119029199f;
__device__ constexpr float kC2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f, -1.0925484305920792f,
                          0.5462742152960396f};
__device__ constexpr float kC3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f, 0.3731763325901154f,
                          -0.4570457994644658f, 1.445305721320277f, -0.5900435899266435f};

// Rest basis function k of sh.slang:25-51 (k in 0..14, in its order) at the
// unit direction (x, y, z); k is a constant wherever these are called (the
// callers' loops are unrolled), so each call is a short polynomial.
__device__ __forceinline__ float sh_basis_at(int k, float x, float y, float z) {
    const float xx = x * x, yy = y * y, zz = z * z;
    switch (k) {
        case 0: return -kC1 * y;
        case 1: return kC1 * z;
        case 2: return -kC1 * x;
        case 3: return kC2[0] * x * y;
        case 4: return kC2[1] * y * z;
        case 5: return kC2[2] * (2.0f * zz - xx - yy);
        case 6: return kC2[3] * x * z;
        case 7: return kC2[4] * (xx - yy);
        case 8: return kC3[0] * y * (3.0f * xx - yy);
        case 9: return kC3[1] * x * y * z;
        case 10: return kC3[2] * y * (4.0f * zz - xx - yy);
        case 11: return kC3[3] * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
        case 12: return kC3[4] * x * (4.0f * zz - xx - yy);
        case 13: return kC3[5] * z * (xx - yy);
        default: return kC3[6] * x * (xx - 3.0f * yy);
    }
}

// The same function and its gradient (d/dx, d/dy, d/dz).
__device__ __forceinline__ void sh_basis_grad_at(int k, float x, float y, float z, float& b, float& gx, float& gy,
                                                 float& gz) {
    const float xx = x * x, yy = y * y, zz = z * z;
    b = sh_basis_at(k, x, y, z);
    gx = gy = gz = 0.0f;
    switch (k) {
        case 0: gy = -kC1; break;
        case 1: gz = kC1; break;
        case 2: gx = -kC1; break;
        case 3: gx = kC2[0] * y; gy = kC2[0] * x; break;
        case 4: gy = kC2[1] * z; gz = kC2[1] * y; break;
        case 5: gx = -2.0f * kC2[2] * x; gy = -2.0f * kC2[2] * y; gz = 4.0f * kC2[2] * z; break;
        case 6: gx = kC2[3] * z; gz = kC2[3] * x; break;
        case 7: gx = 2.0f * kC2[4] * x; gy = -2.0f * kC2[4] * y; break;
        case 8: gx = 6.0f * kC3[0] * x * y; gy = kC3[0] * (3.0f * xx - 3.0f * yy); break;
        case 9: gx = kC3[1] * y * z; gy = kC3[1] * x * z; gz = kC3[1] * x * y; break;
        case 10: gx = -2.0f * kC3[2] * x * y; gy = kC3[2] * (4.0f * zz - xx - 3.0f * yy); gz = 8.0f * kC3[2] * y * z; break;
        case 11:
            gx = -6.0f * kC3[3] * x * z; gy = -6.0f * kC3[3] * y * z; gz = kC3[3] * (6.0f * zz - 3.0f * xx - 3.0f * yy);
            break;
        case 12: gx = kC3[4] * (4.0f * zz - 3.0f * xx - yy); gy = -2.0f * kC3[4] * x * y; gz = 8.0f * kC3[4] * x * z; break;
        case 13: gx = 2.0f * kC3[5] * x * z; gy = -2.0f * kC3[5] * y * z; gz = kC3[5] * (xx - yy); break;
        default: gx = kC3[6] * (3.0f * xx - 3.0f * yy); gy = -6.0f * kC3[6] * x * y; break;
    }
}

// A splat's partials summed in a fixed order. Splats with few pairs are summed
// by their own lane; the warp then sums each splat with more than kSolo pairs
// together (lane l takes pairs l, l + 32, ..., then a butterfly over the
// lanes), so a splat that touches hundreds of tiles does not hold its warp
// for hundreds of dependent iterations.
constexpr uint32_t kSolo = 16;

__device__ __forceinline__ void sum_partials(const float4* __restrict__ part, uint32_t n, float (&g)[9]) {
#pragma unroll 4
    for (uint32_t k = 0; k < n; ++k) {
        const float4 a = __ldg(part + 3 * k), b = __ldg(part + 3 * k + 1), c = __ldg(part + 3 * k + 2);
        g[0] += a.x; g[1] += a.y; g[2] += a.z; g[3] += a.w;
        g[4] += b.x; g[5] += b.y; g[6] += b.z; g[7] += b.w;
        g[8] += c.x;
    }
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// One view's gradients of splat i from its summed partials g: the per-view
// means, log-scale, quaternion and logit gradients added into gm, gls, gq,
// glog (which the caller zeroes), and the 48 SH gradients handed to
// sink(q, value) in coefficient order.
template <class ShSink>
__device__ __forceinline__ void view_grads(const FrameParams& f, uint32_t i, const float* __restrict__ means,
                                           const float* __restrict__ logScales, const float* __restrict__ quats,
                                           const float* __restrict__ logits, const uint16_t* __restrict__ sh,
                                           const float (&g)[9], float (&gm)[3], float (&gls)[3], float (&gq)[4],
                                           float& glog, ShSink&& sink) {
    const float gcx = g[0], gcy = g[1], gA = g[2], gB = g[3], gC = g[4], gAlpha = g[5];

    // ---- forward intermediates ------------------------------------------
    const float px = means[3 * i], py = means[3 * i + 1], pz = means[3 * i + 2];
    const float sig = 1.0f / (1.0f + lrt_exp(-logits[i]));
    const float s0 = lrt_exp(logScales[3 * i]), s1 = lrt_exp(logScales[3 * i + 1]), s2 = lrt_exp(logScales[3 * i + 2]);
    const float qw0 = quats[4 * i], qx0 = quats[4 * i + 1], qy0 = quats[4 * i + 2], qz0 = quats[4 * i + 3];
    const float len = sqrtf(qw0 * qw0 + qx0 * qx0 + qy0 * qy0 + qz0 * qz0);
    const bool unitQ = len > 0.0f;
    const float x = unitQ ? qx0 / len : 0.0f, y = unitQ ? qy0 / len : 0.0f, z = unitQ ? qz0 / len : 0.0f,
                w = unitQ ? qw0 / len : 1.0f;
    const float3 t = to_view(f, make_float3(px, py, pz));
    const float R[3][3] = {{1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y - w * z), 2.0f * (x * z + w * y)},
                           {2.0f * (x * y + w * z), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z - w * x)},
                           {2.0f * (x * z - w * y), 2.0f * (y * z + w * x), 1.0f - 2.0f * (x * x + y * y)}};
    const float S[3] = {s0, s1, s2};
    float M[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) M[a][b] = R[a][b] * S[b];
    const float W[3][3] = {{f.m[0], f.m[1], f.m[2]}, {f.m[4], f.m[5], f.m[6]}, {f.m[8], f.m[9], f.m[10]}};
    float jx0, jx2, jy1, jy2;
    bool clampX = false, clampY = false;
    float limX = 0.0f, limY = 0.0f;
    const float invZ = 1.0f / t.z;
    if (f.ortho) {
        jx0 = f.focalX; jx2 = 0.0f; jy1 = f.focalY; jy2 = 0.0f;
    } else {
        const float limLoX = (-0.15f * static_cast<float>(f.width) - f.centreX) / f.focalX;
        const float limHiX = (1.15f * static_cast<float>(f.width) - f.centreX) / f.focalX;
        const float limLoY = (-0.15f * static_cast<float>(f.height) - f.centreY) / f.focalY;
        const float limHiY = (1.15f * static_cast<float>(f.height) - f.centreY) / f.focalY;
        const float ux = t.x * invZ, uy = t.y * invZ;
        clampX = ux < limLoX || ux > limHiX;
        clampY = uy < limLoY || uy > limHiY;
        limX = ux < limLoX ? limLoX : limHiX;
        limY = uy < limLoY ? limLoY : limHiY;
        const float tx = clampf(ux, limLoX, limHiX) * t.z;
        const float ty = clampf(uy, limLoY, limHiY) * t.z;
        jx0 = f.focalX * invZ; jx2 = -f.focalX * tx * invZ * invZ;
        jy1 = f.focalY * invZ; jy2 = -f.focalY * ty * invZ * invZ;
    }
    float T2x[3], T2y[3], ax[3], ay[3];
    for (int c = 0; c < 3; ++c) {
        T2x[c] = jx0 * W[0][c] + jx2 * W[2][c];
        T2y[c] = jy1 * W[1][c] + jy2 * W[2][c];
    }
    for (int c = 0; c < 3; ++c) {
        ax[c] = T2x[0] * M[0][c] + T2x[1] * M[1][c] + T2x[2] * M[2][c];
        ay[c] = T2y[0] * M[0][c] + T2y[1] * M[1][c] + T2y[2] * M[2][c];
    }
    const float ap = ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2];
    const float bp = ax[0] * ay[0] + ax[1] * ay[1] + ax[2] * ay[2];
    const float cp = ay[0] * ay[0] + ay[1] * ay[1] + ay[2] * ay[2];
    const float detB = ap * cp - bp * bp;
    const float a = ap + 0.3f, c = cp + 0.3f, b = bp;
    const float det = a * c - b * b;
    const float aa = f.antialias != 0 ? sqrtf(fmaxf(detB, 0.0f) / det) : 1.0f;
    const float QA = c / det, QB = -b / det, QC = a / det;

    // ---- colour ---------------------------------------------------------------
    // The fp16 coefficients stay packed (24 words, read as six 16-byte
    // vectors) and are unpacked where used; each basis function and its
    // gradient is formed where it is used, in two passes over the 15 rest
    // functions (the rest sum, then the gradients), so that no 48-value
    // arrays are held at once.
    uint32_t cw[24];
    {
        const uint4* rv = reinterpret_cast<const uint4*>(sh + static_cast<size_t>(i) * 48);
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const uint4 w4 = __ldg(rv + q);
            cw[4 * q] = w4.x;
            cw[4 * q + 1] = w4.y;
            cw[4 * q + 2] = w4.z;
            cw[4 * q + 3] = w4.w;
        }
    }
    auto coef = [&](int q) { return (q & 1) != 0 ? high_half(cw[q >> 1]) : low_half(cw[q >> 1]); };
    float vx = px - f.eye[0], vy = py - f.eye[1], vz = pz - f.eye[2];
    const float vl = sqrtf(vx * vx + vy * vy + vz * vz);
    const float dirx = vx / vl, diry = vy / vl, dirz = vz / vl;
    const uint32_t degree = min(3u, f.shLimit);   // basis functions above it are 0
    const int used = degree == 0 ? 0 : degree == 1 ? 3 : degree == 2 ? 8 : 15;
    constexpr float kSH0 = 0.28209479177387814f;
    float rest[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 15; ++k) {
        if (k < used) {
            const float b = sh_basis_at(k, dirx, diry, dirz);
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) rest[ch] += b * coef(3 + 3 * k + ch);
        }
    }
    // colour = max(base + rest, 0): no gradient where clamped. Basis
    // functions above the evaluated degree are 0, so their coefficients get 0.
    float gcol[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        const float base = 0.5f + kSH0 * coef(ch);
        gcol[ch] = base + rest[ch] > 0.0f ? g[6 + ch] : 0.0f;
        sink(ch, kSH0 * gcol[ch]);
    }
    float gdx = 0.0f, gdy = 0.0f, gdz = 0.0f;
#pragma unroll
    for (int k = 0; k < 15; ++k) {
        float b = 0.0f, bx = 0.0f, by = 0.0f, bz = 0.0f;
        if (k < used) sh_basis_grad_at(k, dirx, diry, dirz, b, bx, by, bz);
        float cg = 0.0f;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            sink(3 + 3 * k + ch, b * gcol[ch]);
            cg += coef(3 + 3 * k + ch) * gcol[ch];
        }
        gdx += cg * bx;
        gdy += cg * by;
        gdz += cg * bz;
    }
    {   // dir = v / |v|, v = p - eye
        const float dotd = gdx * dirx + gdy * diry + gdz * dirz;
        gm[0] += (gdx - dotd * dirx) / vl;
        gm[1] += (gdy - dotd * diry) / vl;
        gm[2] += (gdz - dotd * dirz) / vl;
    }

    // ---- alpha0 = sigmoid(logit) * aa -----------------------------------------
    glog = gAlpha * aa * sig * (1.0f - sig);
    const float gAA = gAlpha * sig;
    float gDetB = 0.0f, gDet = 0.0f;
    if (f.antialias != 0 && detB > 0.0f && aa > 0.0f) {
        gDetB = gAA / (2.0f * aa * det);
        gDet = -gAA * aa / (2.0f * det);
    }

    // ---- conic = inverse of [[a, b], [b, c]] ------------------------------------
    // G_Sigma = -Q G_Q Q with G_Q = [[gA, gB/2], [gB/2, gC]]
    const float h = 0.5f * gB;
    const float t00 = gA * QA + h * QB, t01 = gA * QB + h * QC;
    const float t10 = h * QA + gC * QB, t11 = h * QB + gC * QC;
    const float gS00 = -(QA * t00 + QB * t10), gS01 = -(QA * t01 + QB * t11);
    const float gS11 = -(QB * t01 + QC * t11);
    float ga = gS00 + gDet * c + gDetB * cp;
    float gc = gS11 + gDet * a + gDetB * ap;
    float gb = 2.0f * gS01 - gDet * 2.0f * b - gDetB * 2.0f * bp;

    // ---- a' = ax.ax, b' = ax.ay, c' = ay.ay --------------------------------
    float gax[3], gay[3];
    for (int k = 0; k < 3; ++k) {
        gax[k] = 2.0f * ga * ax[k] + gb * ay[k];
        gay[k] = gb * ax[k] + 2.0f * gc * ay[k];
    }
    // ax = T2x M, ay = T2y M
    float gT2x[3], gT2y[3], gM[3][3];
    for (int r = 0; r < 3; ++r) {
        gT2x[r] = gax[0] * M[r][0] + gax[1] * M[r][1] + gax[2] * M[r][2];
        gT2y[r] = gay[0] * M[r][0] + gay[1] * M[r][1] + gay[2] * M[r][2];
        for (int cc = 0; cc < 3; ++cc) gM[r][cc] = T2x[r] * gax[cc] + T2y[r] * gay[cc];
    }
    // M = R diag(S)
    float gR[3][3];
    for (int cc = 0; cc < 3; ++cc) {
        float gs = 0.0f;
        for (int r = 0; r < 3; ++r) {
            gR[r][cc] = gM[r][cc] * S[cc];
            gs += gM[r][cc] * R[r][cc];
        }
        gls[cc] = gs * S[cc];
    }
    // R(x, y, z, w)
    const float gx = 2.0f * (gR[0][1] * y + gR[0][2] * z + gR[1][0] * y - 2.0f * gR[1][1] * x - gR[1][2] * w +
                             gR[2][0] * z + gR[2][1] * w - 2.0f * gR[2][2] * x);
    const float gy = 2.0f * (-2.0f * gR[0][0] * y + gR[0][1] * x + gR[0][2] * w + gR[1][0] * x + gR[1][2] * z -
                             gR[2][0] * w + gR[2][1] * z - 2.0f * gR[2][2] * y);
    const float gz = 2.0f * (-2.0f * gR[0][0] * z - gR[0][1] * w + gR[0][2] * x + gR[1][0] * w -
                             2.0f * gR[1][1] * z + gR[1][2] * y + gR[2][0] * x + gR[2][1] * y);
    const float gw = 2.0f * (-gR[0][1] * z + gR[0][2] * y + gR[1][0] * z - gR[1][2] * x - gR[2][0] * y +
                             gR[2][1] * x);
    if (unitQ) {   // q_n = q / |q|
        const float dq = gx * x + gy * y + gz * z + gw * w;
        gq[0] = (gw - dq * w) / len;
        gq[1] = (gx - dq * x) / len;
        gq[2] = (gy - dq * y) / len;
        gq[3] = (gz - dq * z) / len;
    }
    // T2 = J W
    float gjx0 = 0.0f, gjx2 = 0.0f, gjy1 = 0.0f, gjy2 = 0.0f;
    for (int cc = 0; cc < 3; ++cc) {
        gjx0 += gT2x[cc] * W[0][cc];
        gjx2 += gT2x[cc] * W[2][cc];
        gjy1 += gT2y[cc] * W[1][cc];
        gjy2 += gT2y[cc] * W[2][cc];
    }
    float gt[3] = {0.0f, 0.0f, 0.0f};
    if (f.ortho) {
        gt[0] += gcx * f.focalX;
        gt[1] += gcy * f.focalY;
    } else {
        // centre = focal t.xy / t.z + c
        gt[0] += gcx * f.focalX * invZ;
        gt[1] += gcy * f.focalY * invZ;
        gt[2] += -(gcx * f.focalX * t.x + gcy * f.focalY * t.y) * invZ * invZ;
        // J: jx0 = fx / tz, jx2 = -fx tx_c / tz^2 (tx_c = t.x, or lim tz when clamped)
        gt[2] += -(gjx0 * f.focalX + gjy1 * f.focalY) * invZ * invZ;
        if (clampX) {
            gt[2] += gjx2 * f.focalX * limX * invZ * invZ;
        } else {
            gt[0] += -gjx2 * f.focalX * invZ * invZ;
            gt[2] += 2.0f * gjx2 * f.focalX * t.x * invZ * invZ * invZ;
        }
        if (clampY) {
            gt[2] += gjy2 * f.focalY * limY * invZ * invZ;
        } else {
            gt[1] += -gjy2 * f.focalY * invZ * invZ;
            gt[2] += 2.0f * gjy2 * f.focalY * t.y * invZ * invZ * invZ;
        }
    }
    // t = W p + t0
    for (int k = 0; k < 3; ++k) gm[k] += W[0][k] * gt[0] + W[1][k] * gt[1] + W[2][k] * gt[2];
}

// The partials of one splat in a frame (its touched count `count` of pairs
// from pair `firstRaw` of `partials`; both 0 for a dead lane), summed into g;
// every lane of the warp takes part. nOut comes back 0 for a dead lane or a
// pair range outside the buffer.
__device__ __forceinline__ void splat_partials(uint32_t count, uint32_t firstRaw, uint32_t lane,
                                               const float* __restrict__ partials, uint32_t partialPairs,
                                               float (&g)[9], uint32_t& nOut) {
    uint32_t n = count;
    const uint32_t first = n != 0 ? firstRaw : 0u;
    // Reads stay inside the partials buffer even for a frame whose pairs
    // overflowed their buffer (the host reports that frame as an error).
    n = first >= partialPairs ? 0u : min(n, partialPairs - first);
#pragma unroll
    for (int q = 0; q < 9; ++q) g[q] = 0.0f;
    const float4* part4 = reinterpret_cast<const float4*>(partials);
    if (n <= kSolo) sum_partials(part4 + static_cast<size_t>(first) * 3, n, g);
    uint32_t many = __ballot_sync(0xFFFFFFFFu, n > kSolo);
    while (many != 0) {
        const int owner = __ffs(many) - 1;
        many &= many - 1;
        const uint32_t on = __shfl_sync(0xFFFFFFFFu, n, owner);
        const uint32_t of = __shfl_sync(0xFFFFFFFFu, first, owner);
        float h[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const float4* p = part4 + static_cast<size_t>(of) * 3;
        for (uint32_t k = lane; k < on; k += 32) {
            const float4 a = __ldg(p + 3 * k), b = __ldg(p + 3 * k + 1), c = __ldg(p + 3 * k + 2);
            h[0] += a.x; h[1] += a.y; h[2] += a.z; h[3] += a.w;
            h[4] += b.x; h[5] += b.y; h[6] += b.z; h[7] += b.w;
            h[8] += c.x;
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
#pragma unroll
            for (int q = 0; q < 9; ++q) h[q] += __shfl_xor_sync(0xFFFFFFFFu, h[q], d);
        }
        if (static_cast<int>(lane) == owner) {
#pragma unroll
            for (int q = 0; q < 9; ++q) g[q] = h[q];
        }
    }
    nOut = n;
}

// One frame: every splat's gradients written (zero for a splat the frame
// does not touch).
template <bool kChained>
__global__ void __launch_bounds__(kThreads, 5)
splat_backward_kernel(FrameParams f, const float* __restrict__ means, const float* __restrict__ logScales,
                      const float* __restrict__ quats, const float* __restrict__ logits,
                      const uint16_t* __restrict__ sh, const uint32_t* __restrict__ touched,
                      const uint32_t* __restrict__ offsets, const float* __restrict__ partials,
                      uint32_t partialPairs, float* __restrict__ gMeans, float* __restrict__ gLogScales,
                      float* __restrict__ gQuats, float* __restrict__ gLogits, float* __restrict__ gSh) {
    chained_entry<kChained>();
    __shared__ float sGsh[48][kThreads];
    const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    const bool live = i < f.count;
    const uint32_t slot = f.base + i;
    // The parameters and SH row are read only after the partials are summed;
    // ask for them now (into L2, no registers held), so their DRAM latency
    // overlaps the count, offset and partial loads that each wait on the last.
    if (live) {
        prefetch_l2(means + 3 * static_cast<size_t>(i));
        prefetch_l2(logScales + 3 * static_cast<size_t>(i));
        prefetch_l2(quats + 4 * static_cast<size_t>(i));
        prefetch_l2(logits + i);
        prefetch_l2(sh + 48 * static_cast<size_t>(i));
        prefetch_l2(sh + 48 * static_cast<size_t>(i) + 40);
    }
    float g[9];
    uint32_t n = 0;
    const uint32_t count = live ? touched[slot] : 0u;
    const uint32_t firstRaw = live ? offsets[slot] : 0u;   // loaded beside the count, not after it
    splat_partials(count, firstRaw, lane, partials, partialPairs, g, n);
    if (!live) return;
    float gm[3] = {0, 0, 0}, gls[3] = {0, 0, 0}, gq[4] = {0, 0, 0, 0}, glog = 0.0f;
    float* gshRow = gSh + static_cast<size_t>(i) * 48;
    if (n == 0) {
        float4* out = reinterpret_cast<float4*>(gshRow);
#pragma unroll
        for (int q = 0; q < 12; ++q) out[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else {
        // The 48 SH gradients go through shared memory (a column per thread)
        // rather than registers, then out as 16-byte stores.
        view_grads(f, i, means, logScales, quats, logits, sh, g, gm, gls, gq, glog,
                   [&](int q, float v) { sGsh[q][threadIdx.x] = v; });
        float4* out = reinterpret_cast<float4*>(gshRow);
#pragma unroll
        for (int q = 0; q < 12; ++q)
            out[q] = make_float4(sGsh[4 * q][threadIdx.x], sGsh[4 * q + 1][threadIdx.x], sGsh[4 * q + 2][threadIdx.x],
                                 sGsh[4 * q + 3][threadIdx.x]);
    }
    for (int k = 0; k < 3; ++k) {
        gMeans[3 * i + k] = gm[k];
        gLogScales[3 * i + k] = gls[k];
    }
    for (int k = 0; k < 4; ++k) gQuats[4 * i + k] = gq[k];
    gLogits[i] = glog;
}

// A chunk of views in one pass. Per splat, view after view in order, the
// view's gradients (view_grads, as above) are added to running sums -- the
// 48 SH ones in shared memory, a column per thread -- and the sums written
// once at the end, so the gradient buffers are read and written once a chunk
// rather than once a view. The sums start from what the buffers hold when
// `accumulate` is set (a batch's later chunks), else from zero: the same
// float additions, in the same order, as a view-by-view pass adding each
// view to the buffers. touched / offsets: one array of `count` per view.
__global__ void __launch_bounds__(kThreads, 3)
splat_backward_views_kernel(const FrameParams* __restrict__ frames, uint32_t views, uint32_t count,
                            const float* __restrict__ means, const float* __restrict__ logScales,
                            const float* __restrict__ quats, const float* __restrict__ logits,
                            const uint16_t* __restrict__ sh, const uint32_t* __restrict__ touched,
                            const uint32_t* __restrict__ offsets, const float* __restrict__ partials,
                            uint32_t partialPairs, float* __restrict__ gMeans, float* __restrict__ gLogScales,
                            float* __restrict__ gQuats, float* __restrict__ gLogits, float* __restrict__ gSh,
                            uint32_t accumulate) {
    __shared__ float sAcc[48][kThreads];
    __shared__ FrameParams sF[kMaxChunkViews];
    {
        const uint32_t words = views * static_cast<uint32_t>(sizeof(FrameParams) / 4);
        const uint32_t* src = reinterpret_cast<const uint32_t*>(frames);
        uint32_t* dst = reinterpret_cast<uint32_t*>(sF);
        for (uint32_t w = threadIdx.x; w < words; w += kThreads) dst[w] = src[w];
    }
    const uint32_t tid = threadIdx.x;
    const uint32_t i = blockIdx.x * kThreads + tid;
    const uint32_t lane = tid & 31u;
    const bool live = i < count;
    float am[3] = {0, 0, 0}, als[3] = {0, 0, 0}, aq[4] = {0, 0, 0, 0}, alog = 0.0f;
    float4* shRow = reinterpret_cast<float4*>(gSh + static_cast<size_t>(i) * 48);
    if (live && accumulate != 0) {
        for (int k = 0; k < 3; ++k) {
            am[k] = gMeans[3 * i + k];
            als[k] = gLogScales[3 * i + k];
        }
        for (int k = 0; k < 4; ++k) aq[k] = gQuats[4 * i + k];
        alog = gLogits[i];
#pragma unroll
        for (int q = 0; q < 12; ++q) {
            const float4 v = shRow[q];
            sAcc[4 * q][tid] = v.x;
            sAcc[4 * q + 1][tid] = v.y;
            sAcc[4 * q + 2][tid] = v.z;
            sAcc[4 * q + 3][tid] = v.w;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 48; ++q) sAcc[q][tid] = 0.0f;
    }
    __syncthreads();
    // The next view's count and first pair are loaded, and its first partials
    // asked into L2, while this view's gradients are computed.
    uint32_t nextCount = live ? touched[sF[0].base + i] : 0u;
    uint32_t nextFirst = live ? offsets[sF[0].base + i] : 0u;
    for (uint32_t v = 0; v < views; ++v) {
        const FrameParams& f = sF[v];
        const uint32_t thisCount = nextCount, thisFirst = nextFirst;
        if (v + 1 < views && live) {
            const size_t at = static_cast<size_t>(v + 1) * count + sF[v + 1].base + i;
            nextCount = touched[at];
            nextFirst = offsets[at];
        }
        float g[9];
        uint32_t n = 0;
        splat_partials(thisCount, thisFirst, lane, partials, partialPairs, g, n);
        if (v + 1 < views && nextCount != 0 && nextFirst < partialPairs) {
            const size_t at = static_cast<size_t>(nextFirst) * kGradStrideFloats;
            prefetch_l2(partials + at);
            if (nextCount > 1 && at + 32 < static_cast<size_t>(partialPairs) * kGradStrideFloats)
                prefetch_l2(partials + at + 32);
        }
        if (!live || n == 0) continue;
        float gm[3] = {0, 0, 0}, gls[3] = {0, 0, 0}, gq[4] = {0, 0, 0, 0}, glog = 0.0f;
        view_grads(f, i, means, logScales, quats, logits, sh, g, gm, gls, gq, glog,
                   [&](int q, float x) { sAcc[q][tid] = __fadd_rn(sAcc[q][tid], x); });
        // The running sums are plain rounded additions (never fused with the
        // product that formed a term), so that they equal the single-view
        // gradients summed in view order.
        for (int k = 0; k < 3; ++k) {
            am[k] = __fadd_rn(am[k], gm[k]);
            als[k] = __fadd_rn(als[k], gls[k]);
        }
        for (int k = 0; k < 4; ++k) aq[k] = __fadd_rn(aq[k], gq[k]);
        alog = __fadd_rn(alog, glog);
    }
    if (!live) return;
    for (int k = 0; k < 3; ++k) {
        gMeans[3 * i + k] = am[k];
        gLogScales[3 * i + k] = als[k];
    }
    for (int k = 0; k < 4; ++k) gQuats[4 * i + k] = aq[k];
    gLogits[i] = alog;
#pragma unroll
    for (int q = 0; q < 12; ++q)
        shRow[q] = make_float4(sAcc[4 * q][tid], sAcc[4 * q + 1][tid], sAcc[4 * q + 2][tid], sAcc[4 * q + 3][tid]);
}

}  // namespace

cudaError_t launch_splat_backward_views(const FrameParams* framesDev, uint32_t views, uint32_t count,
                                        const float* means, const float* logScales, const float* quats,
                                        const float* logits, const uint16_t* sh, const uint32_t* touched,
                                        const uint32_t* offsets, const float* partials, uint32_t partialPairs,
                                        float* gMeans, float* gLogScales, float* gQuats, float* gLogits, float* gSh,
                                        bool accumulate, cudaStream_t stream) {
    if (views > kMaxChunkViews) return cudaErrorInvalidValue;
    if (count == 0 || views == 0) return cudaSuccess;
    const uint32_t blocks = (count + kThreads - 1) / kThreads;
    splat_backward_views_kernel<<<blocks, kThreads, 0, stream>>>(
        framesDev, views, count, means, logScales, quats, logits, sh, touched, offsets, partials, partialPairs, gMeans,
        gLogScales, gQuats, gLogits, gSh, accumulate ? 1u : 0u);
    return cudaGetLastError();
}

cudaError_t launch_splat_backward(const FrameParams& f, const float* means, const float* logScales, const float* quats,
                                  const float* logits, const uint16_t* sh, const uint32_t* touched,
                                  const uint32_t* offsets, const float* partials, uint32_t partialPairs,
                                  float* gMeans, float* gLogScales, float* gQuats, float* gLogits, float* gSh,
                                  cudaStream_t stream) {
    if (f.count == 0) return cudaSuccess;
    const uint32_t blocks = (f.count + kThreads - 1) / kThreads;
    return launch_chained(splat_backward_kernel<true>, splat_backward_kernel<false>, dim3(blocks), dim3(kThreads), 0, stream, f, means, logScales, quats,
                          logits, sh, touched, offsets, partials, partialPairs, gMeans, gLogScales, gQuats, gLogits,
                          gSh);
}

}  // namespace lrt
