// Levels of detail on the device: the build (LodBuilder::build,
// modules/lod/src/Lod.cpp:86-300) and the per-frame cut (CutSelector::select,
// Lod.cpp:349-547). The method is the reference's (shaders/lrt/lod/
// lod_common.slang:1-33, after Kerbl et al. 2024): splats in Morton order, a
// level-r octree cell = a code's top 3r bits, so each cell's splats are one
// run; per cell the additive moments W, S1, S2, C of its splats, turned back
// into one Gaussian; a cell is drawn merged when it projects to at most
// `threshold` pixels and its parent does not, a splat when its finest merged
// cell does not.
//
// What differs is the schedule:
//   * The reference finds each level's groups with a boundary pass, a prefix
//     sum and a host read, one level at a time (Lod.cpp:151-198). A splat
//     begins a group at level r exactly when its code and its predecessor's
//     differ in their top 3r bits, i.e. when the highest differing bit lies
//     in triple t >= 10 - r. So one pass (fused into the reorder) histograms
//     the first level 10 - t at which each splat begins a group, and every
//     level's group count is a running sum of it: one host read in all.
//   * Only the finest stored level's groups are found over the splats; each
//     coarser level's are found over the finer level's cells (its parent
//     codes), a pass over groups rather than splats.
//   * The cut is one kernel per instance over every merged Gaussian (levels
//     coarsest first) and then every splat: each thread decides its item
//     (lod_cut.slang), the block scans the decisions, takes its base by
//     decoupled look-back and gathers its drawn items into the frame's cloud
//     -- the reference's select, prefix sum, count read and gather passes
//     (Lod.cpp:430-514) in one launch, in the same output order.
//
// Arithmetic is restated expression for expression and the library is built
// with -fmad=false, so the merged Gaussians and the cut agree bit for bit with
// the CPU restatement.
#include "kernels.cuh"
#include "lookback.cuh"
#include "raster_common.cuh"

namespace lrt {
namespace {

constexpr uint32_t kLodThreads = 256;
constexpr uint32_t kBoundsBlocks = 148 * 2;
constexpr uint32_t kMomentThreads = 64;

__device__ __forceinline__ float saturate_unit(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// morton.slang:23-28: 10 bits an axis, x in the highest bit of each triple.
__device__ __forceinline__ uint32_t interleave_bits(uint32_t x, uint32_t y, uint32_t z) {
    uint32_t code = 0;
#pragma unroll
    for (uint32_t b = 0; b < 10; ++b)
        code |= (((x >> b) & 1u) << (3 * b + 2)) | (((y >> b) & 1u) << (3 * b + 1)) | (((z >> b) & 1u) << (3 * b));
    return code;
}

// morton.slang:30-33: one axis of a level-`bits` cell code (axisShift 2 for x,
// 1 for y, 0 for z).
__device__ __forceinline__ uint32_t axis_bits(uint32_t cell, uint32_t axisShift, uint32_t bits) {
    uint32_t v = 0;
    for (uint32_t b = 0; b < bits; ++b) v |= ((cell >> (3 * b + axisShift)) & 1u) << b;
    return v;
}

__device__ __forceinline__ uint32_t quantise_axis(float v, float lo, float extent) {
    return min(static_cast<uint32_t>(saturate_unit((v - lo) / extent) * 1024.0f), 1023u);
}

// ------------------------------------------------------------- bounds ------
// CloudLoader::boundsOf (GpuClouds.cpp:93-125; bounds_chunks.slang,
// bounds_reduce.slang): the min and max of the positions. Both are exact, so
// the order of the reduction does not matter.
__global__ void __launch_bounds__(kLodThreads)
lod_bounds_partial_kernel(const float4* __restrict__ positions, uint32_t count, float* __restrict__ partial) {
    __shared__ float sLo[3][kLodThreads / 32], sHi[3][kLodThreads / 32];
    float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (uint32_t i = blockIdx.x * kLodThreads + threadIdx.x; i < count; i += gridDim.x * kLodThreads) {
        const float4 p = __ldg(positions + i);
        lo[0] = fminf(lo[0], p.x), lo[1] = fminf(lo[1], p.y), lo[2] = fminf(lo[2], p.z);
        hi[0] = fmaxf(hi[0], p.x), hi[1] = fmaxf(hi[1], p.y), hi[2] = fmaxf(hi[2], p.z);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xFFFFFFFFu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xFFFFFFFFu, hi[k], o));
        }
        if ((threadIdx.x & 31u) == 0) sLo[k][threadIdx.x >> 5] = lo[k], sHi[k][threadIdx.x >> 5] = hi[k];
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        float l = 3.4e38f, h = -3.4e38f;
        for (uint32_t w = 0; w < kLodThreads / 32; ++w) l = fminf(l, sLo[threadIdx.x][w]), h = fmaxf(h, sHi[threadIdx.x][w]);
        partial[blockIdx.x * 6 + threadIdx.x] = l;
        partial[blockIdx.x * 6 + 3 + threadIdx.x] = h;
    }
}

// The cloud's bounds (the caller's when given) and the cubic extent of
// Lod.cpp:91-97: the largest edge, at least 1e-6, times 1.0001 so the far
// corner quantises inside the last cell.
__global__ void __launch_bounds__(kLodThreads)
lod_bounds_final_kernel(const float* __restrict__ partial, uint32_t blocks, const float* __restrict__ given,
                        LodGlobals* __restrict__ g) {
    __shared__ float sLo[3][kLodThreads / 32], sHi[3][kLodThreads / 32];
    float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (uint32_t b = threadIdx.x; given == nullptr && b < blocks; b += kLodThreads) {
#pragma unroll
        for (int k = 0; k < 3; ++k) lo[k] = fminf(lo[k], partial[b * 6 + k]), hi[k] = fmaxf(hi[k], partial[b * 6 + 3 + k]);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xFFFFFFFFu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xFFFFFFFFu, hi[k], o));
        }
        if ((threadIdx.x & 31u) == 0) sLo[k][threadIdx.x >> 5] = lo[k], sHi[k][threadIdx.x >> 5] = hi[k];
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    float extent = 0.0f;
    for (int k = 0; k < 3; ++k) {
        float l = 3.4e38f, h = -3.4e38f;
        if (given != nullptr) {
            l = given[k], h = given[3 + k];
        } else {
            for (uint32_t w = 0; w < kLodThreads / 32; ++w) l = fminf(l, sLo[k][w]), h = fmaxf(h, sHi[k][w]);
        }
        g->lo[k] = l, g->hi[k] = h;
        const float edge = h - l;
        extent = extent < edge ? edge : extent;
    }
    extent = extent < 1e-6f ? 1e-6f : extent;
    g->extent = extent * 1.0001f;
}

// ------------------------------------------------------------- Morton ------
// lod_morton.slang:12-20: each splat's code, and the identity order the sort
// carries along.
__global__ void __launch_bounds__(kLodThreads)
lod_morton_kernel(const float4* __restrict__ positions, uint32_t count, const LodGlobals* __restrict__ g,
                  uint32_t* __restrict__ keys, uint32_t* __restrict__ order) {
    const uint32_t i = blockIdx.x * kLodThreads + threadIdx.x;
    if (i >= count) return;
    const float extent = fmaxf(g->extent, 1e-20f);
    const float4 p = __ldg(positions + i);
    keys[i] = interleave_bits(quantise_axis(p.x, g->lo[0], extent), quantise_axis(p.y, g->lo[1], extent),
                              quantise_axis(p.z, g->lo[2], extent));
    order[i] = i;
}

// ------------------------------------------------------------ reorder ------
// lod_reorder.slang:18-31 (slot k takes splat order[k]), fused with the
// level histogram: the first level at which splat k begins a group.
// A warp copies its 32 rows of harmonics together, lane by word, so a row's
// words are read and written by consecutive lanes.
__global__ void __launch_bounds__(kLodThreads)
lod_reorder_kernel(const uint32_t* __restrict__ order, const uint32_t* __restrict__ codes, uint32_t count,
                   uint32_t shWords, const float4* __restrict__ srcPositions, const uint4* __restrict__ srcShape,
                   const uint32_t* __restrict__ srcSh, LodSplatArrays store, LodGlobals* __restrict__ g) {
    __shared__ uint32_t sHist[kLodLevels + 2];
    if (threadIdx.x < kLodLevels + 2) sHist[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t k = blockIdx.x * kLodThreads + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t mine = k < count ? __ldg(order + k) : 0u;
    if (k < count) {
        store.positions[k] = __ldg(srcPositions + mine);
        store.shape[k] = __ldg(srcShape + mine);
        if (k > 0) {
            const uint32_t x = __ldg(codes + k) ^ __ldg(codes + k - 1);
            const uint32_t level = x == 0 ? kLodLevels + 1 : kLodLevels - (31u - __clz(x)) / 3u;
            atomicAdd(&sHist[level], 1u);
        }
    }
    const uint32_t warpFirst = k - lane;
    if (shWords > 0 && warpFirst < count) {   // warp-uniform
        const uint32_t rows = min(32u, count - warpFirst);
        const uint32_t words = rows * shWords;
        for (uint32_t base = 0; base < words; base += 32) {
            const uint32_t w = base + lane;
            const uint32_t row = min(w / shWords, 31u);
            const uint32_t src = __shfl_sync(0xFFFFFFFFu, mine, row);
            if (w < words)
                store.sh[static_cast<size_t>(warpFirst) * shWords + w] =
                    __ldg(srcSh + static_cast<size_t>(src) * shWords + (w - row * shWords));
        }
    }
    __syncthreads();
    if (threadIdx.x < kLodLevels + 2 && sHist[threadIdx.x] != 0) atomicAdd(&g->firstLevel[threadIdx.x], sHist[threadIdx.x]);
}

// ------------------------------------------------------------- groups ------
// lod_boundaries.slang + lod_groups.slang for the finest stored level, in one
// compaction: splat k begins a group when its level-`level` cell differs from
// its predecessor's; group g's first splat and cell code are written by it.
__global__ void __launch_bounds__(kLodThreads)
lod_finest_groups_kernel(const uint32_t* __restrict__ codes, uint32_t count, uint32_t shift, uint32_t capacity,
                         uint32_t* __restrict__ starts, uint32_t* __restrict__ cells, uint64_t* __restrict__ status,
                         uint32_t* __restrict__ ticket, uint32_t* __restrict__ total, uint32_t* __restrict__ err) {
    __shared__ uint32_t sPart, sBase;
    __shared__ uint32_t sWarp[kLodThreads / 32];
    if (threadIdx.x == 0) sPart = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t part = sPart;
    const uint32_t k = part * kLodThreads + threadIdx.x;
    uint32_t cell = 0;
    bool begins = false;
    if (k < count) {
        cell = __ldg(codes + k) >> shift;
        begins = k == 0 || (__ldg(codes + k - 1) >> shift) != cell;
    }
    uint32_t blockTotal = 0;
    const uint32_t local = block_scan<kLodThreads>(begins ? 1u : 0u, sWarp, &blockTotal);
    const uint32_t lastPart = (count + kLodThreads - 1) / kLodThreads - 1;
    const uint32_t base = block_base(part, lastPart, blockTotal, status, total, err, &sBase);
    // capacity: the count the level histogram gave; the host checks the two agree.
    if (!begins || base + local >= capacity) return;
    starts[base + local] = k;
    cells[base + local] = cell;
}

// A coarser level's groups from the finer level's: fine group h begins a
// coarse group when its parent cell (code >> 3) differs from h - 1's. The
// coarse group's cell, and its first child (the children of group g are the
// fine groups firstChild[g] .. firstChild[g + 1] - 1, the run
// lod_merge_moments.slang:21-23 finds through its first splat).
__global__ void __launch_bounds__(kLodThreads)
lod_parent_groups_kernel(const uint32_t* __restrict__ fineCells, uint32_t fineCount, uint32_t capacity,
                         uint32_t* __restrict__ cells,
                         uint32_t* __restrict__ firstChild, uint64_t* __restrict__ status,
                         uint32_t* __restrict__ ticket, uint32_t* __restrict__ total, uint32_t* __restrict__ err) {
    __shared__ uint32_t sPart, sBase;
    __shared__ uint32_t sWarp[kLodThreads / 32];
    if (threadIdx.x == 0) sPart = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t part = sPart;
    const uint32_t h = part * kLodThreads + threadIdx.x;
    uint32_t parent = 0;
    bool begins = false;
    if (h < fineCount) {
        parent = __ldg(fineCells + h) >> 3;
        begins = h == 0 || (__ldg(fineCells + h - 1) >> 3) != parent;
    }
    uint32_t blockTotal = 0;
    const uint32_t local = block_scan<kLodThreads>(begins ? 1u : 0u, sWarp, &blockTotal);
    const uint32_t lastPart = (fineCount + kLodThreads - 1) / kLodThreads - 1;
    const uint32_t base = block_base(part, lastPart, blockTotal, status, total, err, &sBase);
    if (!begins || base + local >= capacity) return;
    cells[base + local] = parent;
    firstChild[base + local] = h;
}

// ------------------------------------------------------------ moments ------
// lod_leaf_moments.slang:26-64: the finest stored level's moments, each
// group's splats summed in order by one thread (the reference's order, so
// the sums round alike). With w = opacity x the area of the splat's two
// longest axes: W, S1 = w mu, S2 = w (Sigma + mu mu^T) as xx xy xz yy yz zz,
// C = w base colour, then w times each rest coefficient.
template <uint32_t kKeep>
__global__ void __launch_bounds__(kMomentThreads)
lod_leaf_moments_kernel(LodSplatArrays store, uint32_t count, uint32_t shWords, const uint32_t* __restrict__ starts,
                        uint32_t groups, float* __restrict__ moments) {
    constexpr uint32_t kStride = kLodMomentsHead + 3 * kKeep;
    const uint32_t g = blockIdx.x * kMomentThreads + threadIdx.x;
    if (g >= groups) return;
    // Clamped to the splats (the starts are checked on the host afterwards).
    const uint32_t first = min(__ldg(starts + g), count);
    const uint32_t end = min(g + 1 < groups ? __ldg(starts + g + 1) : count, count);
    float acc[kStride];
#pragma unroll
    for (uint32_t k = 0; k < kStride; ++k) acc[k] = 0.0f;
    for (uint32_t i = first; i < end; ++i) {
        const float4 p = store.positions[i];
        const uint4 w = store.shape[i];
        const float sx = lrt_exp(low_half(w.y)), sy = lrt_exp(high_half(w.y)), sz = lrt_exp(low_half(w.z));
        float x, y, z, qw;
        decode_rotation_word(w.x, x, y, z, qw);
        const float r[3][3] = {
            {1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y - qw * z), 2.0f * (x * z + qw * y)},
            {2.0f * (x * y + qw * z), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z - qw * x)},
            {2.0f * (x * z - qw * y), 2.0f * (y * z + qw * x), 1.0f - 2.0f * (x * x + y * y)}};
        const float s[3] = {sx, sy, sz};
        float m[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) m[a][b] = r[a][b] * s[b];
        auto cov = [&](int a, int b) { return m[a][0] * m[b][0] + m[a][1] * m[b][1] + m[a][2] * m[b][2]; };
        const float smallest = fminf(fminf(sx, sy), sz);
        const float area = sx * sy * sz / fmaxf(smallest, 1e-20f);
        const float weight = p.w * area;
        acc[0] = acc[0] + weight;
        acc[1] = acc[1] + weight * p.x;
        acc[2] = acc[2] + weight * p.y;
        acc[3] = acc[3] + weight * p.z;
        acc[4] = acc[4] + weight * (cov(0, 0) + p.x * p.x);
        acc[5] = acc[5] + weight * (cov(0, 1) + p.x * p.y);
        acc[6] = acc[6] + weight * (cov(0, 2) + p.x * p.z);
        acc[7] = acc[7] + weight * (cov(1, 1) + p.y * p.y);
        acc[8] = acc[8] + weight * (cov(1, 2) + p.y * p.z);
        acc[9] = acc[9] + weight * (cov(2, 2) + p.z * p.z);
        acc[10] = acc[10] + weight * high_half(w.z);
        acc[11] = acc[11] + weight * low_half(w.w);
        acc[12] = acc[12] + weight * high_half(w.w);
        const uint32_t* row = store.sh + static_cast<size_t>(i) * shWords;
#pragma unroll
        for (uint32_t h = 0; h < 3 * kKeep; ++h) {
            const uint32_t word = row[h / 2];
            acc[kLodMomentsHead + h] = acc[kLodMomentsHead + h] + weight * ((h & 1u) != 0 ? high_half(word) : low_half(word));
        }
    }
    float* out = moments + static_cast<size_t>(g) * kStride;
#pragma unroll
    for (uint32_t k = 0; k < kStride; ++k) out[k] = acc[k];
}

// lod_merge_moments.slang:19-31: a coarser group's moments, its children's
// summed in child order. One thread per (group, moment), moments fastest, so
// a warp's loads of one child's row are contiguous; each sum still runs over
// the children in order, as the reference's per-group loop does.
__global__ void __launch_bounds__(kLodThreads)
lod_merge_moments_kernel(const uint32_t* __restrict__ firstChild, uint32_t groups, uint32_t fineGroups,
                         const float* __restrict__ fine, float* __restrict__ moments, uint32_t stride) {
    const size_t t = static_cast<size_t>(blockIdx.x) * kLodThreads + threadIdx.x;
    if (t >= static_cast<size_t>(groups) * stride) return;
    const uint32_t g = static_cast<uint32_t>(t / stride);
    const uint32_t k = static_cast<uint32_t>(t - static_cast<size_t>(g) * stride);
    const uint32_t first = min(__ldg(firstChild + g), fineGroups);
    const uint32_t end = min(g + 1 < groups ? __ldg(firstChild + g + 1) : fineGroups, fineGroups);
    float sum = 0.0f;
    for (uint32_t h = first; h < end; ++h) sum = sum + __ldg(fine + static_cast<size_t>(h) * stride + k);
    moments[t] = sum;
}

// ----------------------------------------------------------- finalize ------
// o = a b, each entry summed over k in order.
__device__ __forceinline__ void mat3_mul(const float a[3][3], const float b[3][3], float o[3][3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) o[r][c] = a[r][0] * b[0][c] + a[r][1] * b[1][c] + a[r][2] * b[2][c];
}

// o = a^T b.
__device__ __forceinline__ void mat3_tmul(const float a[3][3], const float b[3][3], float o[3][3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) o[r][c] = a[0][r] * b[0][c] + a[1][r] * b[1][c] + a[2][r] * b[2][c];
}

__device__ __forceinline__ float sign_of(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }

// lod_finalize.slang:16-40: cyclic Jacobi, six sweeps over (0,1), (0,2),
// (1,2); `a` ends diagonal and v's columns are the eigenvectors. Each
// rotation is applied as the full products J^T (A J) and V J.
__device__ __forceinline__ void jacobi3(float a[3][3], float v[3][3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) v[r][c] = r == c ? 1.0f : 0.0f;
#pragma unroll 1
    for (int sweep = 0; sweep < 6; ++sweep) {
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0;
            const int q = pq == 0 ? 1 : 2;
            const float apq = a[p][q];
            if (fabsf(apq) < 1e-30f) continue;
            const float theta = (a[q][q] - a[p][p]) / (2.0f * apq);
            const float t = sign_of(theta + 1e-30f) / (fabsf(theta) + sqrtf(theta * theta + 1.0f));
            const float c = 1.0f / sqrtf(t * t + 1.0f);
            const float s = t * c;
            float j[3][3] = {{1.0f, 0.0f, 0.0f}, {0.0f, 1.0f, 0.0f}, {0.0f, 0.0f, 1.0f}};
            j[p][p] = c;
            j[q][q] = c;
            j[p][q] = s;
            j[q][p] = -s;
            float b[3][3], o[3][3];
            mat3_mul(a, j, b);
            mat3_tmul(j, b, a);
            mat3_mul(v, j, o);
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) v[r][cc] = o[r][cc];
        }
    }
}

// packing.slang:76-93: the quaternion (x, y, z, w) of a rotation whose
// columns are the axes, normalised.
__device__ __forceinline__ float4 quaternion_of_axes(const float m[3][3]) {
    const float trace = m[0][0] + m[1][1] + m[2][2];
    float x, y, z, w;
    if (trace > 0.0f) {
        const float s = 0.5f / sqrtf(trace + 1.0f);
        x = (m[2][1] - m[1][2]) * s, y = (m[0][2] - m[2][0]) * s, z = (m[1][0] - m[0][1]) * s, w = 0.25f / s;
    } else if (m[0][0] > m[1][1] && m[0][0] > m[2][2]) {
        const float s = 2.0f * sqrtf(1.0f + m[0][0] - m[1][1] - m[2][2]);
        x = 0.25f * s, y = (m[1][0] + m[0][1]) / s, z = (m[0][2] + m[2][0]) / s, w = (m[2][1] - m[1][2]) / s;
    } else if (m[1][1] > m[2][2]) {
        const float s = 2.0f * sqrtf(1.0f - m[0][0] + m[1][1] - m[2][2]);
        x = (m[1][0] + m[0][1]) / s, y = 0.25f * s, z = (m[2][1] + m[1][2]) / s, w = (m[0][2] - m[2][0]) / s;
    } else {
        const float s = 2.0f * sqrtf(1.0f - m[0][0] - m[1][1] + m[2][2]);
        x = (m[0][2] + m[2][0]) / s, y = (m[2][1] + m[1][2]) / s, z = 0.25f * s, w = (m[1][0] - m[0][1]) / s;
    }
    const float l = sqrtf(x * x + y * y + z * z + w * w);
    return make_float4(x / l, y / l, z / l, w / l);
}

// lod_finalize.slang:42-96: moments to one packed Gaussian per group, every
// stored level in one launch (the levels' moments are contiguous).
__global__ void __launch_bounds__(kMomentThreads)
lod_finalize_kernel(const float* __restrict__ moments, uint32_t groups, uint32_t keep, uint32_t shWords,
                    LodSplatArrays out) {
    const uint32_t g = blockIdx.x * kMomentThreads + threadIdx.x;
    if (g >= groups) return;
    const uint32_t stride = kLodMomentsHead + 3 * keep;
    const float* at = moments + static_cast<size_t>(g) * stride;
    const float weight = fmaxf(at[0], 1e-30f);
    const float mu[3] = {at[1] / weight, at[2] / weight, at[3] / weight};
    float a[3][3] = {{at[4] / weight, at[5] / weight, at[6] / weight},
                     {at[5] / weight, at[7] / weight, at[8] / weight},
                     {at[6] / weight, at[8] / weight, at[9] / weight}};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) a[r][c] = a[r][c] - mu[r] * mu[c];
    float axes[3][3];
    jacobi3(a, axes);
    const float det = axes[0][0] * (axes[1][1] * axes[2][2] - axes[1][2] * axes[2][1]) -
                      axes[0][1] * (axes[1][0] * axes[2][2] - axes[1][2] * axes[2][0]) +
                      axes[0][2] * (axes[1][0] * axes[2][1] - axes[1][1] * axes[2][0]);
    if (det < 0.0f) {
        axes[0][2] = -axes[0][2];
        axes[1][2] = -axes[1][2];
        axes[2][2] = -axes[2][2];
    }
    const float s[3] = {sqrtf(fmaxf(a[0][0], 1e-14f)), sqrtf(fmaxf(a[1][1], 1e-14f)), sqrtf(fmaxf(a[2][2], 1e-14f))};
    const float smallest = fminf(fminf(s[0], s[1]), s[2]);
    const float area = s[0] * s[1] * s[2] / fmaxf(smallest, 1e-20f);
    const float opacity = fminf(at[0] / fmaxf(area, 1e-30f), 0.99f);
    const float base[3] = {at[10] / weight, at[11] / weight, at[12] / weight};
    out.positions[g] = make_float4(mu[0], mu[1], mu[2], opacity);
    const float ls[3] = {lrt_log(s[0]), lrt_log(s[1]), lrt_log(s[2])};
    out.shape[g] = make_uint4(encode_quaternion(quaternion_of_axes(axes)), pack_halves(half_safe(ls[0]), half_safe(ls[1])),
                              pack_halves(half_safe(ls[2]), half_safe(base[0])),
                              pack_halves(half_safe(base[1]), half_safe(base[2])));
    // The rest coefficients two halves a word; words past them (a row is at
    // least one word) are zero.
    uint32_t* row = out.sh + static_cast<size_t>(g) * shWords;
    uint32_t word = 0, filled = 0, written = 0;
    for (uint32_t h = 0; h < keep * 3; ++h) {
        const uint32_t bits = float_to_half(half_safe(at[kLodMomentsHead + h] / weight)) & 0xFFFFu;
        word |= bits << (filled * 16);
        if (++filled == 2) {
            row[written++] = word;
            word = 0;
            filled = 0;
        }
    }
    if (filled == 1) row[written++] = word;
    for (; written < shWords; ++written) row[written] = 0u;
}

// ----------------------------------------------------------------- cut -----
// lod_cut.slang:12-30: the pixels a level-`level` cell spans at its nearest
// point to the eye (perspective), or its edge in pixels (orthographic).
__device__ __forceinline__ float projected_edge(const LodCutParams& c, uint32_t cell, uint32_t level) {
    const float edge = c.extent / static_cast<float>(1u << level);
    if (c.ortho != 0) return edge * c.pixelsPerUnit;
    const float lox = c.lo[0] + static_cast<float>(axis_bits(cell, 2, level)) * edge;
    const float loy = c.lo[1] + static_cast<float>(axis_bits(cell, 1, level)) * edge;
    const float loz = c.lo[2] + static_cast<float>(axis_bits(cell, 0, level)) * edge;
    const float dx = fminf(fmaxf(c.eye[0], lox), lox + edge) - c.eye[0];
    const float dy = fminf(fmaxf(c.eye[1], loy), loy + edge) - c.eye[1];
    const float dz = fminf(fmaxf(c.eye[2], loz), loz + edge) - c.eye[2];
    const float distance = fmaxf(sqrtf(dx * dx + dy * dy + dz * dz), 1e-6f);
    return edge * c.pixelsPerUnit / distance;
}

__device__ __forceinline__ bool cell_small(const LodCutParams& c, uint32_t cell, uint32_t level) {
    return c.threshold > 0.0f && projected_edge(c, cell, level) <= c.threshold;
}

constexpr uint32_t kCutItems = 4;                        // consecutive items per thread
constexpr uint32_t kCutTile = kLodThreads * kCutItems;   // items per block
constexpr uint32_t kCutMaskWords = kCutTile / 32;

// Whether item j of the cut is drawn (lodCutGroups / lodCutFinest /
// lodCutSplats, lod_cut.slang:32-86, every chunk resident): a merged
// Gaussian when its cell is small and its parent's is not (or it is on the
// coarsest stored level), a splat when its finest-level cell is not small.
__device__ __forceinline__ bool cut_drawn(const LodCutParams& c, uint32_t j, uint32_t key) {
    if (j < c.merged) {
        // The stored level holding j (constant indices keep the table in the
        // parameter bank).
        uint32_t level = 0;
#pragma unroll
        for (uint32_t l = 1; l <= kLodLevels; ++l) level += (l < c.levels && j >= c.levelBase[l]) ? 1u : 0u;
        const uint32_t octree = c.coarsest + level;
        const bool here = cell_small(c, key, octree);
        const bool above = level > 0 && cell_small(c, key >> 3, octree - 1);
        return here && !above;
    }
    const uint32_t finest = c.coarsest + c.levels - 1;
    return !cell_small(c, key >> (3 * (kLodLevels - finest)), finest);
}

// The cut in three passes, none waiting on another block. Items: the merged
// Gaussians, stored levels coarsest first, then the splats (the reference's
// output order, Lod.cpp:486-514). First every block decides its 1024 items
// (four consecutive a thread, their cell or code loads in flight together)
// and writes them as a 32-word bitmask and a count.
__global__ void __launch_bounds__(kLodThreads)
lod_cut_decide_kernel(LodCutParams c, const uint32_t* __restrict__ cells, const uint32_t* __restrict__ codes,
                      uint32_t* __restrict__ flags, uint32_t* __restrict__ blockCounts) {
    __shared__ uint32_t sMask[kCutMaskWords];
    __shared__ uint32_t sWarp[kLodThreads / 32];
    if (threadIdx.x < kCutMaskWords) sMask[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t items = c.merged + c.count;
    const uint32_t j0 = blockIdx.x * kCutTile + threadIdx.x * kCutItems;
    uint32_t key[kCutItems];
#pragma unroll
    for (uint32_t i = 0; i < kCutItems; ++i) {
        const uint32_t j = j0 + i;
        key[i] = j < c.merged ? __ldg(cells + j) : (j < items ? __ldg(codes + (j - c.merged)) : 0u);
    }
    uint32_t f = 0;
#pragma unroll
    for (uint32_t i = 0; i < kCutItems; ++i)
        if (j0 + i < items && cut_drawn(c, j0 + i, key[i])) f |= 1u << i;
    if (f != 0) atomicOr(&sMask[threadIdx.x >> 3], f << ((threadIdx.x & 7u) * kCutItems));
    const uint32_t n = __reduce_add_sync(0xFFFFFFFFu, static_cast<uint32_t>(__popc(f)));
    if ((threadIdx.x & 31u) == 0) sWarp[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x < kCutMaskWords) flags[static_cast<size_t>(blockIdx.x) * kCutMaskWords + threadIdx.x] = sMask[threadIdx.x];
    if (threadIdx.x == 0) {
        uint32_t total = 0;
        for (uint32_t w = 0; w < kLodThreads / 32; ++w) total += sWarp[w];
        blockCounts[blockIdx.x] = total;
    }
}

// Then the tiles' counts become their first output slots (one block; integer
// sums, so the order does not matter), and the last one the drawn total.
constexpr uint32_t kCutScanThreads = 1024;
__global__ void __launch_bounds__(kCutScanThreads)
lod_cut_bases_kernel(const uint32_t* __restrict__ blockCounts, uint32_t tiles, uint32_t* __restrict__ tileBase,
                     uint32_t* __restrict__ counts) {
    __shared__ uint32_t sWarp[kCutScanThreads / 32];
    uint32_t carry = 0;
    for (uint32_t at = 0; at < tiles; at += kCutScanThreads) {
        const uint32_t t = at + threadIdx.x;
        const uint32_t v = t < tiles ? blockCounts[t] : 0u;
        uint32_t total = 0;
        const uint32_t ex = block_scan<kCutScanThreads>(v, sWarp, &total);
        if (t < tiles) tileBase[t] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) counts[0] = carry;
}

// Last, every 256 items gather their drawn records (lod_gather.slang:18-33):
// the tile's first slot plus the drawn items of the tile's earlier quarters
// give the block's base; a ballot per warp and a block scan rank its items,
// listed in order in shared memory; consecutive threads copy consecutive
// outputs, the harmonics rows word by word. Drawn items past `capacity` are
// counted, not written. counts[1] gets the merged Gaussians drawn (the rank
// of the first splat item).
constexpr uint32_t kCutGather = kLodThreads;   // items per gather block
__global__ void __launch_bounds__(kLodThreads)
lod_cut_gather_kernel(LodCutParams c, const uint32_t* __restrict__ flags, const uint32_t* __restrict__ tileBase,
                      LodSplatArrays merged, LodSplatArrays store, LodSplatArrays out,
                      uint32_t* __restrict__ counts) {
    __shared__ uint32_t sWarp[kLodThreads / 32];
    __shared__ uint32_t sItem[kCutGather];
    constexpr uint32_t kQuarters = kCutTile / kCutGather;
    constexpr uint32_t kQuarterWords = kCutGather / 32;
    const uint32_t tile = blockIdx.x / kQuarters, quarter = blockIdx.x % kQuarters;
    const uint32_t* mask = flags + static_cast<size_t>(tile) * kCutMaskWords;
    uint32_t earlier = 0;   // drawn items of the tile's earlier quarters
    for (uint32_t w = 0; w < quarter * kQuarterWords; ++w) earlier += static_cast<uint32_t>(__popc(__ldg(mask + w)));
    const uint32_t base = __ldg(tileBase + tile) + earlier;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t bits = __ldg(mask + quarter * kQuarterWords + (threadIdx.x >> 5));
    const bool drawn = (bits >> lane) & 1u;
    const uint32_t j = blockIdx.x * kCutGather + threadIdx.x;
    uint32_t blockTotal = 0;
    const uint32_t local = block_scan<kLodThreads>(drawn ? 1u : 0u, sWarp, &blockTotal);
    if (j == c.merged) counts[1] = base + local;
    if (drawn) sItem[local] = j;
    __syncthreads();
    const uint32_t room = c.capacity > base ? min(blockTotal, c.capacity - base) : 0u;
    for (uint32_t r = threadIdx.x; r < room; r += kLodThreads) {
        const uint32_t o = base + r;
        const uint32_t item = sItem[r];
        const bool isMerged = item < c.merged;
        const uint32_t k = isMerged ? item : item - c.merged;
        out.positions[o] = isMerged ? merged.positions[k] : store.positions[k];
        out.shape[o] = isMerged ? merged.shape[k] : store.shape[k];
    }
    if (c.shWords == 0) return;
    const uint32_t words = room * c.shWords;
    for (uint32_t w = threadIdx.x; w < words; w += kLodThreads) {
        const uint32_t r = w / c.shWords;
        const uint32_t col = w - r * c.shWords;
        const uint32_t item = sItem[r];
        const uint32_t* src = item < c.merged ? merged.sh + static_cast<size_t>(item) * c.shWords
                                              : store.sh + static_cast<size_t>(item - c.merged) * c.shWords;
        out.sh[static_cast<size_t>(base + r) * c.shWords + col] = src[col];
    }
}

uint32_t blocks_for(uint32_t n, uint32_t threads) { return (n + threads - 1) / threads; }

}  // namespace

size_t lod_bounds_partial_bytes() { return size_t{kBoundsBlocks} * 6 * sizeof(float); }
uint32_t lod_compaction_threads() { return kLodThreads; }

cudaError_t launch_lod_bounds(const float4* positions, uint32_t count, const float* given, LodGlobals* globals,
                              float* partial, cudaStream_t stream) {
    uint32_t blocks = 0;
    if (given == nullptr) {
        blocks = std::max<uint32_t>(1u, std::min(kBoundsBlocks, blocks_for(count, kLodThreads)));
        lod_bounds_partial_kernel<<<blocks, kLodThreads, 0, stream>>>(positions, count, partial);
    }
    lod_bounds_final_kernel<<<1, kLodThreads, 0, stream>>>(partial, blocks, given, globals);
    return cudaGetLastError();
}

cudaError_t launch_lod_morton(const float4* positions, uint32_t count, const LodGlobals* globals, uint32_t* keys,
                              uint32_t* order, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    lod_morton_kernel<<<blocks_for(count, kLodThreads), kLodThreads, 0, stream>>>(positions, count, globals, keys, order);
    return cudaGetLastError();
}

cudaError_t launch_lod_reorder(const uint32_t* order, const uint32_t* codes, uint32_t count, uint32_t shWords,
                               const float4* srcPositions, const uint4* srcShape, const uint32_t* srcSh,
                               LodSplatArrays store, LodGlobals* globals, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    lod_reorder_kernel<<<blocks_for(count, kLodThreads), kLodThreads, 0, stream>>>(
        order, codes, count, shWords, srcPositions, srcShape, srcSh, store, globals);
    return cudaGetLastError();
}

cudaError_t launch_lod_finest_groups(const uint32_t* codes, uint32_t count, uint32_t level, uint32_t capacity,
                                     uint32_t* starts, uint32_t* cells, void* status, uint32_t* total, uint32_t* err,
                                     cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    const uint32_t blocks = blocks_for(count, kLodThreads);
    uint64_t* words = static_cast<uint64_t*>(status);
    uint32_t* ticket = reinterpret_cast<uint32_t*>(words + blocks);
    lod_finest_groups_kernel<<<blocks, kLodThreads, 0, stream>>>(codes, count, 3 * (kLodLevels - level), capacity,
                                                                  starts, cells, words, ticket, total, err);
    return cudaGetLastError();
}

cudaError_t launch_lod_parent_groups(const uint32_t* fineCells, uint32_t fineCount, uint32_t capacity,
                                     uint32_t* cells, uint32_t* firstChild, void* status, uint32_t* total,
                                     uint32_t* err, cudaStream_t stream) {
    if (fineCount == 0) return cudaSuccess;
    const uint32_t blocks = blocks_for(fineCount, kLodThreads);
    uint64_t* words = static_cast<uint64_t*>(status);
    uint32_t* ticket = reinterpret_cast<uint32_t*>(words + blocks);
    lod_parent_groups_kernel<<<blocks, kLodThreads, 0, stream>>>(fineCells, fineCount, capacity, cells, firstChild,
                                                                  words, ticket, total, err);
    return cudaGetLastError();
}

cudaError_t launch_lod_leaf_moments(const LodSplatArrays store, uint32_t count, uint32_t restPerColour,
                                    uint32_t shWords, const uint32_t* starts, uint32_t groups, float* moments,
                                    cudaStream_t stream) {
    if (groups == 0) return cudaSuccess;
    const uint32_t blocks = blocks_for(groups, kMomentThreads);
    switch (restPerColour) {
        case 0: lod_leaf_moments_kernel<0><<<blocks, kMomentThreads, 0, stream>>>(store, count, shWords, starts, groups, moments); break;
        case 3: lod_leaf_moments_kernel<3><<<blocks, kMomentThreads, 0, stream>>>(store, count, shWords, starts, groups, moments); break;
        case 8: lod_leaf_moments_kernel<8><<<blocks, kMomentThreads, 0, stream>>>(store, count, shWords, starts, groups, moments); break;
        case 15: lod_leaf_moments_kernel<15><<<blocks, kMomentThreads, 0, stream>>>(store, count, shWords, starts, groups, moments); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_lod_merge_moments(const uint32_t* firstChild, uint32_t groups, uint32_t fineGroups,
                                     const float* fineMoments, float* moments, uint32_t stride, cudaStream_t stream) {
    if (groups == 0) return cudaSuccess;
    const size_t threads = static_cast<size_t>(groups) * stride;
    lod_merge_moments_kernel<<<static_cast<uint32_t>((threads + kLodThreads - 1) / kLodThreads), kLodThreads, 0,
                               stream>>>(firstChild, groups, fineGroups, fineMoments, moments, stride);
    return cudaGetLastError();
}

cudaError_t launch_lod_finalize(const float* moments, uint32_t groups, uint32_t restPerColour, uint32_t shWords,
                                LodSplatArrays merged, cudaStream_t stream) {
    if (groups == 0) return cudaSuccess;
    lod_finalize_kernel<<<blocks_for(groups, kMomentThreads), kMomentThreads, 0, stream>>>(moments, groups,
                                                                                         restPerColour, shWords, merged);
    return cudaGetLastError();
}

size_t lod_cut_scratch_bytes(uint32_t items) {
    const size_t tiles = std::max<uint32_t>(blocks_for(items, kCutTile), 1u);
    return tiles * (kCutMaskWords + 2) * sizeof(uint32_t) + 16;
}

cudaError_t launch_lod_cut(const LodCutParams& c, const uint32_t* cells, const uint32_t* codes,
                           const LodSplatArrays merged, const LodSplatArrays store, LodSplatArrays out,
                           void* scratch, uint32_t* counts, cudaStream_t stream) {
    const uint32_t items = c.merged + c.count;
    if (items == 0) return cudaSuccess;
    const uint32_t tiles = blocks_for(items, kCutTile);
    uint32_t* flags = static_cast<uint32_t*>(scratch);
    uint32_t* tileCounts = flags + size_t{tiles} * kCutMaskWords;
    uint32_t* tileBase = tileCounts + tiles;
    lod_cut_decide_kernel<<<tiles, kLodThreads, 0, stream>>>(c, cells, codes, flags, tileCounts);
    lod_cut_bases_kernel<<<1, kCutScanThreads, 0, stream>>>(tileCounts, tiles, tileBase, counts);
    lod_cut_gather_kernel<<<blocks_for(items, kCutGather), kLodThreads, 0, stream>>>(c, flags, tileBase, merged,
                                                                                     store, out, counts);
    return cudaGetLastError();
}

}  // namespace lrt
