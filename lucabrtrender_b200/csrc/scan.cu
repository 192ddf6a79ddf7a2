// Exclusive prefix sum of uint32 counts: the duplication offsets (stage b)
// and the public lrt_prefix_sum (the reference's gpu::PrefixSum,
// modules/gpu/src/algo/PrefixSum.cpp:58-88, which scans in three dispatches
// with one thread per chunk and a one-thread middle pass).
//
// B200 form: one pass, decoupled look-back. A block takes the next partition
// of 4096 counts (256 threads x 16, 16-byte loads), reduces with warp
// shuffles, publishes its aggregate, then adds its predecessors' published
// values (inclusive ones end the walk). Partitions are handed out by an
// atomic ticket in launch order, so a block only ever waits on blocks that
// are already running; every wait is bounded and raises kErrTimeout instead
// of spinning forever. Sums are 64-bit: a total past 2^32 - 1 raises
// kErrTooManyPairs.
#include "kernels.cuh"
#include "raster_common.cuh"

#include <cuda/atomic>

namespace lrt {
namespace {

constexpr uint32_t kScanThreads = 256;
constexpr uint32_t kScanItems = 16;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;
constexpr uint64_t kFlagAggregate = 1ull << 62;
constexpr uint64_t kFlagInclusive = 2ull << 62;
constexpr uint64_t kValueMask = (1ull << 62) - 1;
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint64_t warp_inclusive_scan(uint64_t v) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint64_t o = __shfl_up_sync(0xFFFFFFFFu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

__global__ void __launch_bounds__(kScanThreads)
scan_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t* __restrict__ total,
            uint32_t n, uint64_t* __restrict__ status, uint32_t* __restrict__ ticket, uint32_t* __restrict__ err) {
    __shared__ uint32_t sPart;
    __shared__ uint64_t sWarp[kScanThreads / 32];
    __shared__ uint64_t sPrefix;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u, warp = tid >> 5;
    if (tid == 0) sPart = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t part = sPart;
    const uint32_t base = part * kScanTile;
    if (base >= n) return;

    // Blocked arrangement: thread t owns counts [base + 16t, base + 16t + 16).
    uint32_t v[kScanItems];
    const uint32_t first = base + tid * kScanItems;
    const bool vec = (reinterpret_cast<uintptr_t>(in) & 15u) == 0 && first + kScanItems <= n;
    if (vec) {
        const uint4* src = reinterpret_cast<const uint4*>(in + first);
#pragma unroll
        for (uint32_t k = 0; k < kScanItems / 4; ++k) {
            const uint4 q = __ldg(src + k);
            v[4 * k] = q.x; v[4 * k + 1] = q.y; v[4 * k + 2] = q.z; v[4 * k + 3] = q.w;
        }
    } else {
#pragma unroll
        for (uint32_t k = 0; k < kScanItems; ++k) v[k] = first + k < n ? in[first + k] : 0u;
    }
    uint64_t mine = 0;
#pragma unroll
    for (uint32_t k = 0; k < kScanItems; ++k) mine += v[k];
    const uint64_t incl = warp_inclusive_scan(mine);
    if (lane == 31) sWarp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < kScanThreads / 32 ? sWarp[lane] : 0;
        w = warp_inclusive_scan(w);
        if (lane < kScanThreads / 32) sWarp[lane] = w;   // inclusive per warp
    }
    __syncthreads();
    const uint64_t blockSum = sWarp[kScanThreads / 32 - 1];
    const uint64_t warpExcl = warp == 0 ? 0 : sWarp[warp - 1];

    if (tid == 0) {
        cuda::atomic_ref<uint64_t, cuda::thread_scope_device> mineStatus(status[part]);
        uint64_t prefix = 0;
        if (part == 0) {
            mineStatus.store(kFlagInclusive | blockSum, cuda::memory_order_relaxed);
        } else {
            mineStatus.store(kFlagAggregate | blockSum, cuda::memory_order_relaxed);
            int64_t p = static_cast<int64_t>(part) - 1;
            uint32_t spins = 0;
            while (p >= 0) {
                cuda::atomic_ref<uint64_t, cuda::thread_scope_device> s(status[p]);
                const uint64_t word = s.load(cuda::memory_order_relaxed);
                if ((word & ~kValueMask) == 0) {
                    if (++spins > kSpinLimit) {
                        atomicOr(err, kErrTimeout);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                prefix += word & kValueMask;
                if (word & kFlagInclusive) break;
                --p;
            }
            mineStatus.store(kFlagInclusive | (prefix + blockSum), cuda::memory_order_relaxed);
        }
        sPrefix = prefix;
        if (base + kScanTile >= n) {
            const uint64_t all = prefix + blockSum;
            if (all > 0xFFFFFFFFull) atomicOr(err, kErrTooManyPairs);
            *total = static_cast<uint32_t>(all);
        }
    }
    __syncthreads();
    uint64_t run = sPrefix + warpExcl + (incl - mine);
    uint32_t o[kScanItems];
#pragma unroll
    for (uint32_t k = 0; k < kScanItems; ++k) {
        o[k] = static_cast<uint32_t>(run);
        run += v[k];
    }
    const bool vecOut = (reinterpret_cast<uintptr_t>(out) & 15u) == 0 && first + kScanItems <= n;
    if (vecOut) {
        uint4* dst = reinterpret_cast<uint4*>(out + first);
#pragma unroll
        for (uint32_t k = 0; k < kScanItems / 4; ++k)
            dst[k] = make_uint4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
    } else {
#pragma unroll
        for (uint32_t k = 0; k < kScanItems; ++k)
            if (first + k < n) out[first + k] = o[k];
    }
}

__device__ __forceinline__ void zero_words(uint32_t* __restrict__ p, size_t words) {
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    // Words before the first 16-byte boundary, then 16-byte stores, then the
    // tail.
    const size_t head = min(words, static_cast<size_t>((16u - (reinterpret_cast<uintptr_t>(p) & 15u)) & 15u) / 4u);
    if (i < head) p[i] = 0u;
    const size_t quads = (words - head) / 4;
    uint4* q = reinterpret_cast<uint4*>(p + head);
    for (size_t k = i; k < quads; k += stride) q[k] = make_uint4(0u, 0u, 0u, 0u);
    const size_t tail = head + quads * 4;
    if (i < words - tail) p[tail + i] = 0u;
}

__global__ void zero_kernel(uint32_t* __restrict__ p, size_t words) { zero_words(p, words); }

struct ZeroList {
    ZeroRegion r[kZeroRegions];
    uint32_t count;
};
template <bool kChained>
__global__ void zero_regions_kernel(ZeroList list) {
    chained_entry<kChained>();
    for (uint32_t k = 0; k < list.count; ++k) zero_words(static_cast<uint32_t*>(list.r[k].p), list.r[k].bytes / 4);
}

uint32_t zero_blocks(size_t bytes) {
    const size_t quads = (bytes / 4 + 3) / 4;
    return static_cast<uint32_t>(std::min<size_t>(std::max<size_t>((quads + 255) / 256, 1), 148 * 8));
}

}  // namespace

cudaError_t launch_zero(void* p, size_t bytes, cudaStream_t stream) {
    if (bytes == 0) return cudaSuccess;
    if ((bytes & 3u) != 0 || (reinterpret_cast<uintptr_t>(p) & 3u) != 0) return cudaErrorInvalidValue;
    zero_kernel<<<zero_blocks(bytes), 256, 0, stream>>>(static_cast<uint32_t*>(p), bytes / 4);
    return cudaGetLastError();
}

cudaError_t launch_zero_regions(const ZeroRegion* regions, uint32_t count, cudaStream_t stream) {
    if (count > kZeroRegions) return cudaErrorInvalidValue;
    ZeroList list{};
    size_t largest = 0;
    for (uint32_t k = 0; k < count; ++k) {
        if ((regions[k].bytes & 3u) != 0 || (reinterpret_cast<uintptr_t>(regions[k].p) & 3u) != 0)
            return cudaErrorInvalidValue;
        list.r[k] = regions[k];
        largest = std::max(largest, regions[k].bytes);
    }
    list.count = count;
    if (largest == 0) return cudaSuccess;
    return launch_chained(zero_regions_kernel<true>, zero_regions_kernel<false>, dim3(zero_blocks(largest)), dim3(256), 0, stream, list);
}

size_t scan_scratch_bytes(uint32_t n) {
    const size_t parts = (static_cast<size_t>(n) + kScanTile - 1) / kScanTile;
    return 16 + std::max<size_t>(parts, 1) * sizeof(uint64_t);
}

cudaError_t launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t* total, uint32_t n,
                                  void* scratch, uint32_t* err, cudaStream_t stream) {
    if (n == 0) return cudaMemsetAsync(total, 0, sizeof(uint32_t), stream);
    const size_t bytes = scan_scratch_bytes(n);
    cudaError_t e = cudaMemsetAsync(scratch, 0, bytes, stream);
    if (e != cudaSuccess) return e;
    uint32_t* ticket = static_cast<uint32_t*>(scratch);
    uint64_t* status = reinterpret_cast<uint64_t*>(static_cast<char*>(scratch) + 16);
    const uint32_t parts = (n + kScanTile - 1) / kScanTile;
    scan_kernel<<<parts, kScanThreads, 0, stream>>>(in, out, total, n, status, ticket, err);
    return cudaGetLastError();
}

}  // namespace lrt
