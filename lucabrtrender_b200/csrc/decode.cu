// Cloud decode on the device: raw records to the packed layout the projection
// reads (CloudLoader::upload, modules/scene/src/GpuClouds.cpp:151-226).
//
// The reference runs three dispatches per slice: validate (a flag per
// record, shaders/lrt/scene/splat_validate.slang:14-29), a prefix sum of the
// flags, and decode (splat_decode.slang:20-91, which writes record i at
// base + dest[i] when it is valid). Here one kernel does all three: a block
// validates its 128 records, scans their flags, takes the count of kept
// records before it from a decoupled look-back over the earlier blocks
// (taken in ticket order), and decodes its kept records straight to their
// places. The decode arithmetic restates splat_encoding.slang:21-115 and
// packing.slang:26-50,104-113 expression for expression; the library is built
// with -fmad=false, so it rounds as the CPU restatement does.
#include "kernels.cuh"
#include "raster_common.cuh"
#include "lookback.cuh"

namespace lrt {
namespace {

constexpr uint32_t kDecodeThreads = 128;   // records a block (smaller blocks: more of them resident)
constexpr uint32_t kPointThreads = 256;
constexpr float kSH0 = 0.28209479177387814f;

__device__ __forceinline__ float field_of(const float* raw, uint32_t record, uint32_t stride, uint32_t field) {
    return raw[static_cast<size_t>(record) * stride + field];
}

__device__ __forceinline__ float decode_opacity(float v, uint32_t mode) {
    if (mode == 0) return 1.0f / (1.0f + lrt_exp(-v));
    if (mode == 2) return v / 255.0f;
    return v;
}

__device__ __forceinline__ float3 decode_position(const float* raw, uint32_t i, const lrt_splat_encoding& e) {
    const uint32_t s = e.floats_per_record;
    const float3 v = make_float3(field_of(raw, i, s, e.x) * e.position_scale, field_of(raw, i, s, e.y) * e.position_scale,
                                 field_of(raw, i, s, e.z) * e.position_scale);
    return e.flip_yz != 0 ? make_float3(v.x, -v.y, -v.z) : v;
}

__device__ __forceinline__ float decode_log_scale(float v, uint32_t mode) {
    if (mode == 2) return v / 16.0f - 10.0f;
    return mode == 0 ? v : lrt_log(fmaxf(v, 1e-30f));
}

// color.slang:21-24
__device__ __forceinline__ float linear_to_srgb(float c) {
    c = fmaxf(c, 0.0f);
    return c <= 0.0031308f ? c * 12.92f : 1.055f * lrt_pow(c, 1.0f / 2.4f) - 0.055f;
}

__device__ __forceinline__ float decode_colour(float v, uint32_t mode) {
    if (mode == 0) return 0.5f + kSH0 * v;
    if (mode == 2) return v / 255.0f;
    if (mode == 3) return 0.5f + kSH0 * ((v / 255.0f - 0.5f) / 0.15f);
    if (mode == 4) return linear_to_srgb(v);
    return v;
}

__device__ __forceinline__ float decode_byte_unit(float v, uint32_t mode) { return mode == 1 ? (v - 128.0f) / 128.0f : v; }

// splat_encoding.slang:80-85: the sign of a rest coefficient under y, z -> -y, -z.
__device__ __forceinline__ float rest_flip_sign(uint32_t basis) {
    constexpr uint32_t kNegative = 0x2D4Bu;   // bases 0 1 3 6 8 10 11 13 are odd in y xor z
    return (kNegative >> min(basis, 14u)) & 1u ? -1.0f : 1.0f;
}

// Rest coefficient h (rgb per basis) of record i, decoded and, under y, z ->
// -y, -z, sign-flipped (splat_decode.slang:68-76, splat_encoding.slang:56-68).
__device__ __forceinline__ uint32_t rest_field(const lrt_splat_encoding& e, uint32_t h) {
    const uint32_t basis = h / 3, colour = h - basis * 3;
    return e.rest_colour_outer != 0 ? e.rest_base + colour * e.rest_per_colour + basis : e.rest_base + h;
}
__device__ __forceinline__ float rest_value(const float* raw, uint32_t i, const lrt_splat_encoding& e, uint32_t h) {
    const float value = decode_byte_unit(field_of(raw, i, e.floats_per_record, rest_field(e, h)), e.rest_mode);
    return e.flip_yz != 0 ? value * rest_flip_sign(h / 3) : value;
}

// splat_encoding.slang:91-126: (x, y, z, w), not yet normalised.
__device__ __forceinline__ float4 decode_quaternion(const float* raw, uint32_t i, const lrt_splat_encoding& e) {
    const uint32_t s = e.floats_per_record;
    float q[4];
    if (e.rotation_mode == 2) {
        const float x = field_of(raw, i, s, e.rot_x) / 127.5f - 1.0f;
        const float y = field_of(raw, i, s, e.rot_y) / 127.5f - 1.0f;
        const float z = field_of(raw, i, s, e.rot_z) / 127.5f - 1.0f;
        q[0] = x;
        q[1] = y;
        q[2] = z;
        q[3] = sqrtf(fmaxf(0.0f, 1.0f - (x * x + y * y + z * z)));
    } else if (e.rotation_mode == 3) {
        uint32_t comp = static_cast<uint32_t>(field_of(raw, i, s, e.rot_x)) |
                        (static_cast<uint32_t>(field_of(raw, i, s, e.rot_y)) << 16);
        const uint32_t largest = comp >> 30;
        q[0] = q[1] = q[2] = q[3] = 0.0f;
        float sum = 0.0f;
#pragma unroll
        for (int k = 3; k >= 0; --k) {
            if (static_cast<uint32_t>(k) == largest) continue;
            const float magnitude = kSqrtHalfF * static_cast<float>(comp & 511u) / 511.0f;
            q[k] = ((comp >> 9) & 1u) != 0 ? -magnitude : magnitude;
            sum = sum + q[k] * q[k];
            comp = comp >> 10;
        }
        const float rest = sqrtf(fmaxf(0.0f, 1.0f - sum));
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (static_cast<uint32_t>(k) == largest) q[k] = rest;
    } else {
        q[0] = decode_byte_unit(field_of(raw, i, s, e.rot_x), e.rotation_mode);
        q[1] = decode_byte_unit(field_of(raw, i, s, e.rot_y), e.rotation_mode);
        q[2] = decode_byte_unit(field_of(raw, i, s, e.rot_z), e.rotation_mode);
        q[3] = decode_byte_unit(field_of(raw, i, s, e.rot_w), e.rotation_mode);
    }
    if (e.flip_yz != 0) return make_float4(q[0], -q[1], -q[2], q[3]);
    return make_float4(q[0], q[1], q[2], q[3]);
}


// splat_decode.slang:30-57: record `at` of `src`, kept, to place j (its
// position, opacity, rotation, scales and base colour).
__device__ __forceinline__ void decode_head(const float* src, uint32_t at, const lrt_splat_encoding& e, float3 p,
                                            float a, float ls0, float ls1, float ls2, uint32_t j,
                                            float4* __restrict__ positions, uint4* __restrict__ shape) {
    const uint32_t s = e.floats_per_record;
    positions[j] = make_float4(p.x, p.y, p.z, fminf(fmaxf(a, 0.0f), 1.0f));
    const float4 q = decode_quaternion(src, at, e);
    const float qLength = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    const uint32_t rotation = encode_quaternion(qLength > 1e-8f ? q : make_float4(0.0f, 0.0f, 0.0f, 1.0f));
    const float b0 = decode_colour(field_of(src, at, s, e.dc0), e.colour_mode);
    const float b1 = decode_colour(field_of(src, at, s, e.dc1), e.colour_mode);
    const float b2 = decode_colour(field_of(src, at, s, e.dc2), e.colour_mode);
    shape[j] = make_uint4(rotation, pack_halves(half_safe(ls0), half_safe(ls1)), pack_halves(half_safe(ls2), half_safe(b0)),
                          pack_halves(half_safe(b1), half_safe(b2)));
}

// splat_decode.slang:58-90: the rest coefficients of record `at`, rgb per
// basis, two halves a word, to `row`; every word of the row is written
// (unused halves zero).
__device__ __forceinline__ void decode_rest_row(const float* src, uint32_t at, const lrt_splat_encoding& e,
                                                uint32_t keep, uint32_t shWords, uint32_t* row) {
    const uint32_t values = keep * 3;
    uint32_t w = 0;
    for (uint32_t h = 0; h < values; h += 2, ++w) {
        const float v0 = rest_value(src, at, e, h);
        const float v1 = h + 1 < values ? rest_value(src, at, e, h + 1) : 0.0f;
        row[w] = pack_halves(half_safe(v0), half_safe(v1));
    }
    for (; w < shWords; ++w) row[w] = 0u;
}

__global__ void __launch_bounds__(kDecodeThreads)
decode_splats_kernel(const float* __restrict__ raw, uint32_t count, lrt_splat_encoding e, uint32_t keep,
                     uint32_t shWords, float4* __restrict__ positions, uint4* __restrict__ shape,
                     uint32_t* __restrict__ sh, uint64_t* __restrict__ status, uint32_t* __restrict__ ticket,
                     uint32_t* __restrict__ total, uint32_t* __restrict__ err, uint32_t stage) {
    extern __shared__ __align__(16) float sRaw[];
    __shared__ uint32_t sPart, sBase;
    __shared__ uint32_t sWarp[kDecodeThreads / 32];
    __shared__ uint32_t sKept[kDecodeThreads];   // the block's kept records, by rank
    if (threadIdx.x == 0) sPart = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t part = sPart;
    const uint32_t i = part * kDecodeThreads + threadIdx.x;
    const bool inRange = i < count;
    const uint32_t s = e.floats_per_record;
    // With `stage`, the block's records (contiguous in memory) are first
    // copied to shared memory with 16-byte asynchronous copies, consecutive
    // threads taking consecutive vectors and every copy issued before the
    // wait (the block's whole slice in flight at once), and each thread then
    // reads its record's fields there rather than 32 scattered lines a warp.
    const float* src = raw;
    uint32_t at = i;
    if (stage != 0) {
        const uint32_t first = part * kDecodeThreads;
        const uint32_t n = min(kDecodeThreads, count - min(first, count));
        const uint32_t floats = n * s;
        const float* g = raw + static_cast<size_t>(first) * s;
        for (uint32_t v = threadIdx.x; v < floats / 4; v += kDecodeThreads) cp_async16(sRaw + v * 4, g + v * 4);
        for (uint32_t f = (floats / 4) * 4 + threadIdx.x; f < floats; f += kDecodeThreads) cp_async4(sRaw + f, g + f);
        cp_async_wait_all();
        __syncthreads();
        src = sRaw;
        at = threadIdx.x;
    }

    // splat_validate.slang:19-28
    bool valid = false;
    float3 p = make_float3(0.0f, 0.0f, 0.0f);
    float a = 0.0f, ls0 = 0.0f, ls1 = 0.0f, ls2 = 0.0f;
    if (inRange) {
        p = decode_position(src, at, e);
        a = decode_opacity(field_of(src, at, s, e.opacity), e.opacity_mode);
        ls0 = decode_log_scale(field_of(src, at, s, e.scale0), e.scale_mode);
        ls1 = decode_log_scale(field_of(src, at, s, e.scale1), e.scale_mode);
        ls2 = decode_log_scale(field_of(src, at, s, e.scale2), e.scale_mode);
        const bool finite = isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(ls0) && isfinite(ls1) &&
                            isfinite(ls2) && fabsf(ls0) < 60.0f && fabsf(ls1) < 60.0f && fabsf(ls2) < 60.0f;
        valid = finite && a >= 1.0f / 255.0f;
    }
    uint32_t blockTotal = 0;
    const uint32_t local = block_scan<kDecodeThreads>(valid ? 1u : 0u, sWarp, &blockTotal);
    const uint32_t lastPart = (count + kDecodeThreads - 1) / kDecodeThreads - 1;
    const uint32_t base = block_base(part, lastPart, blockTotal, status, total, err, &sBase);
    if (valid) {
        decode_head(src, at, e, p, a, ls0, ls1, ls2, base + local, positions, shape);
        if (stage == 0) decode_rest_row(src, at, e, keep, shWords, sh + static_cast<size_t>(base + local) * shWords);
        sKept[local] = threadIdx.x;
    }
    if (stage == 0) return;
    // Staged, the block's kept rows (contiguous in the output) are written a
    // row per warp step, lane w making word w: the lane's two fields and
    // signs are fixed, and each step stores one contiguous row.
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u;
    if (lane >= shWords) return;
    const uint32_t values = keep * 3;
    const uint32_t h0 = 2 * lane, h1 = 2 * lane + 1;
    const uint32_t f0 = rest_field(e, h0), f1 = rest_field(e, h1);
    const float sign0 = rest_flip_sign(h0 / 3), sign1 = rest_flip_sign(h1 / 3);
    uint32_t* out = sh + static_cast<size_t>(base) * shWords + lane;
    for (uint32_t r = threadIdx.x >> 5; r < blockTotal; r += kDecodeThreads / 32) {
        const float* rec = sRaw + sKept[r] * s;
        float v0 = 0.0f, v1 = 0.0f;
        if (h0 < values) {
            v0 = decode_byte_unit(rec[f0], e.rest_mode);
            if (e.flip_yz != 0) v0 = v0 * sign0;
        }
        if (h1 < values) {
            v1 = decode_byte_unit(rec[f1], e.rest_mode);
            if (e.flip_yz != 0) v1 = v1 * sign1;
        }
        out[static_cast<size_t>(r) * shWords] = pack_halves(half_safe(v0), half_safe(v1));
    }
}

// points_validate.slang:19-28 and points_decode.slang:24-41, fused the same way.
__global__ void __launch_bounds__(kPointThreads)
decode_points_kernel(const float* __restrict__ raw, uint32_t count, uint32_t colourKind, float detail,
                     float4* __restrict__ positions, uint2* __restrict__ colours, uint64_t* __restrict__ status,
                     uint32_t* __restrict__ ticket, uint32_t* __restrict__ total, uint32_t* __restrict__ err) {
    __shared__ uint32_t sPart, sBase;
    __shared__ uint32_t sWarp[kPointThreads / 32];
    if (threadIdx.x == 0) sPart = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t part = sPart;
    const uint32_t i = part * kPointThreads + threadIdx.x;
    bool valid = false;
    float r[6] = {0, 0, 0, 0, 0, 0};
    if (i < count) {
        for (int k = 0; k < 6; ++k) r[k] = raw[static_cast<size_t>(i) * 6 + k];
        const uint32_t state = i * 747796405u + 2891336453u;   // hash01, color.slang:30-34
        const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
        const float hash = static_cast<float>((word >> 22u) ^ word) / 4294967295.0f;
        const bool kept = detail >= 1.0f || hash < detail;
        valid = isfinite(r[0]) && isfinite(r[1]) && isfinite(r[2]) && kept;
    }
    uint32_t blockTotal = 0;
    const uint32_t local = block_scan<kPointThreads>(valid ? 1u : 0u, sWarp, &blockTotal);
    const uint32_t lastPart = (count + kPointThreads - 1) / kPointThreads - 1;
    const uint32_t base = block_base(part, lastPart, blockTotal, status, total, err, &sBase);
    if (!valid) return;
    const uint32_t j = base + local;
    positions[j] = make_float4(r[0], r[1], r[2], 1.0f);
    float rgb[3] = {1.0f, 1.0f, 1.0f};
    for (int c = 0; c < 3; ++c) {
        if (colourKind == 1) rgb[c] = srgb_to_linear(r[3 + c] / 255.0f);
        if (colourKind == 2) rgb[c] = r[3 + c];
    }
    colours[j] = make_uint2(pack_halves(rgb[0], rgb[1]), pack_halves(rgb[2], 1.0f));
}

}  // namespace

// A status word per block of the splat or the point decode (the splat
// decode's blocks are the smaller), then the ticket and the total.
size_t decode_status_bytes(uint32_t count) {
    static_assert(kDecodeThreads <= kPointThreads, "the splat decode has the more blocks");
    return size_t{std::max<uint32_t>((count + kDecodeThreads - 1) / kDecodeThreads, 1u)} * sizeof(uint64_t) + 16;
}

// scratch: decode_status_bytes(count) bytes, zeroed by the caller; its last
// 16 bytes hold the ticket and the total.
cudaError_t launch_decode_splats(const float* raw, uint32_t count, const lrt_splat_encoding& e, uint32_t keep,
                                 uint32_t shWords, float4* positions, uint4* shape, uint32_t* sh, void* scratch,
                                 uint32_t* err, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    const uint32_t blocks = (count + kDecodeThreads - 1) / kDecodeThreads;
    uint64_t* status = static_cast<uint64_t*>(scratch);
    uint32_t* tail = reinterpret_cast<uint32_t*>(static_cast<char*>(scratch) + decode_status_bytes(count) - 16);
    // Stage the records through shared memory when a block's fit (and the
    // records start 16-byte aligned); otherwise read them in place.
    const size_t smem = size_t{kDecodeThreads} * e.floats_per_record * sizeof(float);
    const bool stage = smem <= 160 * 1024 && (reinterpret_cast<uintptr_t>(raw) & 15u) == 0;
    if (stage) {
        const cudaError_t a = cudaFuncSetAttribute(decode_splats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(smem));
        if (a != cudaSuccess) return a;
    }
    decode_splats_kernel<<<blocks, kDecodeThreads, stage ? smem : 0, stream>>>(
        raw, count, e, keep, shWords, positions, shape, sh, status, tail, tail + 1, err, stage ? 1u : 0u);
    return cudaGetLastError();
}

cudaError_t launch_decode_points(const float* raw, uint32_t count, uint32_t colourKind, float detail,
                                 float4* positions, uint32_t* colours, void* scratch, uint32_t* err,
                                 cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    const uint32_t blocks = (count + kPointThreads - 1) / kPointThreads;
    uint64_t* status = static_cast<uint64_t*>(scratch);
    uint32_t* tail = reinterpret_cast<uint32_t*>(static_cast<char*>(scratch) + decode_status_bytes(count) - 16);
    decode_points_kernel<<<blocks, kPointThreads, 0, stream>>>(raw, count, colourKind, detail, positions,
                                                                reinterpret_cast<uint2*>(colours), status, tail,
                                                                tail + 1, err);
    return cudaGetLastError();
}

}  // namespace lrt
