// Stream compaction in one pass: a block scans one flag per thread, takes the
// count of flagged items before it from a decoupled look-back over the
// earlier blocks (Merrill & Garland 2016, "Single-pass Parallel Prefix Scan
// with Decoupled Look-back"), and writes its flagged items straight to their
// places. Blocks take their part of the input in ticket order, so every block
// a look-back waits on has already started. Used by the cloud decode and the
// level-of-detail build and cut.
//
// Status words: one uint64 per part, zeroed before the launch; bit 62 marks a
// block's own total, bit 63 the inclusive prefix through it.
#pragma once

#include <cstdint>
#include <cuda/atomic>

#include "raster_common.cuh"

namespace lrt {

constexpr uint64_t kScanFlagAggregate = 1ull << 62;
constexpr uint64_t kScanFlagInclusive = 2ull << 62;
constexpr uint64_t kScanValueMask = (1ull << 62) - 1;
constexpr uint32_t kScanSpinLimit = 1u << 22;

// One block's exclusive scan of a value per thread; *total gets the block's sum.
// sWarp holds kThreads / 32 words.
template <uint32_t kThreads>
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t* sWarp, uint32_t* total) {
    static_assert(kThreads % 32 == 0 && kThreads <= 1024, "whole warps, one block");
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
        uint32_t w = lane < kThreads / 32 ? sWarp[lane] : 0;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, w, d);
            if (lane >= d) w += o;
        }
        if (lane < kThreads / 32) sWarp[lane] = w;
    }
    __syncthreads();
    const uint32_t before = warp == 0 ? 0 : sWarp[warp - 1];
    *total = sWarp[kThreads / 32 - 1];
    __syncthreads();
    return before + x - v;
}

// The flagged items before this block: warp 0 looks back over a window of 32
// earlier blocks at a time, with bounded waits (a wait that runs out raises
// kErrTimeout in *err and counts what it has). Returns the prefix to every
// thread; the last block also writes the grand total.
__device__ __forceinline__ uint32_t block_base(uint32_t part, uint32_t lastPart, uint32_t blockTotal,
                                               uint64_t* status, uint32_t* total, uint32_t* err, uint32_t* sBase) {
    const uint32_t lane = threadIdx.x & 31u;
    if (threadIdx.x < 32) {
        uint64_t prefix = 0;
        if (lane == 0) {
            cuda::atomic_ref<uint64_t, cuda::thread_scope_device> mine(status[part]);
            mine.store((part == 0 ? kScanFlagInclusive : kScanFlagAggregate) | blockTotal,
                       cuda::memory_order_relaxed);
        }
        if (part > 0) {
            int64_t q = static_cast<int64_t>(part) - 1;
            uint32_t spins = 0;
            while (true) {
                const int64_t idx = q - static_cast<int64_t>(lane);
                uint64_t word = kScanFlagInclusive;
                if (idx >= 0) {
                    cuda::atomic_ref<uint64_t, cuda::thread_scope_device> sref(status[idx]);
                    word = sref.load(cuda::memory_order_relaxed);
                }
                const uint32_t inclusive = __ballot_sync(0xFFFFFFFFu, (word & kScanFlagInclusive) != 0);
                const uint32_t empty = __ballot_sync(0xFFFFFFFFu, (word & ~kScanValueMask) == 0);
                const uint32_t first = inclusive != 0 ? static_cast<uint32_t>(__ffs(inclusive)) - 1u : 32u;
                const uint32_t upTo = first < 32u ? (2u << first) - 1u : 0xFFFFFFFFu;
                if ((empty & upTo) != 0) {
                    if (++spins > kScanSpinLimit) {
                        if (lane == 0) atomicOr(err, kErrTimeout);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                uint64_t v = ((upTo >> lane) & 1u) ? (word & kScanValueMask) : 0ull;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
                prefix += v;
                if (first < 32u) break;
                q -= 32;
            }
            if (lane == 0) {
                cuda::atomic_ref<uint64_t, cuda::thread_scope_device> mine(status[part]);
                mine.store(kScanFlagInclusive | (prefix + blockTotal), cuda::memory_order_relaxed);
            }
        }
        if (lane == 0) {
            *sBase = static_cast<uint32_t>(prefix);
            if (part == lastPart && total != nullptr) *total = static_cast<uint32_t>(prefix + blockTotal);
        }
    }
    __syncthreads();
    return *sBase;
}

// Bytes of status words (and the ticket and total after them) for a
// compaction over `count` items, `threads` to a block.
inline size_t compaction_status_bytes(uint32_t count, uint32_t threads) {
    const uint32_t parts = (count + threads - 1) / threads;
    return size_t{parts > 0 ? parts : 1u} * sizeof(uint64_t) + 16;
}

}  // namespace lrt
