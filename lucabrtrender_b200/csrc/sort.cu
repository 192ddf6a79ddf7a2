// Stable LSD radix sort, onesweep form (Adinets & Merrill, "Onesweep: A
// Faster Least Significant Digit Radix Sort for GPUs", 2022), used for the
// rasteriser's pair sort (stage c) and for the public lrt_radix_sort (the
// reference's gpu::RadixSort, modules/gpu/src/algo/RadixSort.cpp:80-157,
// which runs four dispatches per 8-bit pass with one thread walking each
// chunk serially).
//
// Here a sort is one histogram kernel that reads the keys once and counts
// every pass's digits, then one kernel per 8-bit digit that:
//   1. takes the next partition (3072 keys, 4096 in sorts of more than 2^23
//      keys) by atomic ticket (launch order),
//   2. ranks its keys stably inside each warp (the lanes sharing a digit
//      from eight ballots, one per digit bit; a partial last partition is
//      padded with all-ones keys, which sort after every real key;
//      keys are warp-striped, so a warp's item j covers 32 consecutive keys
//      and items are visited in order), and across warps with per-warp
//      digit counts,
//   3. publishes its per-digit counts and resolves the prefix of all earlier
//      partitions by decoupled look-back (bounded waits),
//   4. scatters keys (and values) into shared memory in digit order, then
//      writes them out so that consecutive threads write consecutive slots.
// Only the key bits asked for are sorted: the pass count is ceil(bits / 8).
// Key types: uint32 and uint64, with or without uint32 values. The key count
// is read on the device (at most `cap`), or is `cap` when no count is given.
#include "kernels.cuh"
#include "raster_common.cuh"

#include <cuda/atomic>

namespace lrt {
namespace {

constexpr uint32_t kSortThreads = 256;
constexpr uint32_t kSortWarps = kSortThreads / 32;
constexpr uint32_t kSortItems = 12;
constexpr uint32_t kSortTile = kSortThreads * kSortItems;
// Sorts of more than kLargeKeys keys take kLargeItems keys a thread: fewer,
// longer partitions (measured: the 256M-pair tile sort of a 6M-splat 4K
// frame 5.36 against 5.79 ms), while smaller sorts keep 12 (16 was slower
// for the 1M-slot depth sort).
constexpr uint32_t kLargeItems = 16;
constexpr uint32_t kLargeKeys = 1u << 23;
constexpr uint32_t kLargeTile = kSortThreads * kLargeItems;
constexpr uint32_t kDigits = 256;
// A look-back word holds a digit's running count and, in its top bits, the
// status (aggregate or inclusive). Sorts of fewer than 2^30 keys use 32-bit
// words (30 bits of count); larger ones 64-bit words (a 32-bit count, the
// status in bits 32-33), so no count can spill into the status bits.
template <typename W>
struct LookWord;
template <>
struct LookWord<uint32_t> {
    static constexpr uint32_t kAggregate = 1u << 30, kInclusive = 2u << 30, kValue = (1u << 30) - 1;
};
template <>
struct LookWord<unsigned long long> {
    static constexpr unsigned long long kAggregate = 1ull << 32, kInclusive = 2ull << 32, kValue = 0xFFFFFFFFull;
};
constexpr uint32_t kSmallSortMax = (1u << 30) - 1;   // the most keys 32-bit words can count
constexpr uint32_t kSpinLimit = 1u << 22;
constexpr uint32_t kMaxPasses = 8;
constexpr uint32_t kHistThreads = 512;
constexpr uint32_t kLookWords = 4;   // earlier partitions' status words a look-back step reads

// 256-wide exclusive scan across the block (one value per thread).
__device__ __forceinline__ uint32_t block_exclusive_scan_256(uint32_t v, uint32_t* sWarp) {
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
        uint32_t w = lane < kSortWarps ? sWarp[lane] : 0;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, w, d);
            if (lane >= d) w += o;
        }
        if (lane < kSortWarps) sWarp[lane] = w;
    }
    __syncthreads();
    const uint32_t before = warp == 0 ? 0 : sWarp[warp - 1];
    __syncthreads();
    return before + x - v;
}

// The lanes of the warp holding the same digit d (0..255), from one ballot
// per digit bit.
__device__ __forceinline__ uint32_t match_digit(uint32_t d) {
    uint32_t m = 0xFFFFFFFFu;
#pragma unroll
    for (uint32_t b = 0; b < 8; ++b) {
        const bool bit = ((d >> b) & 1u) != 0;
        const uint32_t v = __ballot_sync(0xFFFFFFFFu, bit);
        m &= bit ? v : ~v;
    }
    return m;
}

template <typename K>
__device__ __forceinline__ uint32_t digit_of(K key, uint32_t shift) {
    return static_cast<uint32_t>(key >> shift) & 0xFFu;
}

template <typename K>
__global__ void __launch_bounds__(kHistThreads)
histogram_kernel(const K* __restrict__ keys, const uint32_t* __restrict__ dCount, uint32_t cap,
                 uint32_t firstBit, uint32_t passes, uint32_t* __restrict__ hist) {
    __shared__ uint32_t sHist[kMaxPasses * kDigits];
    for (uint32_t i = threadIdx.x; i < passes * kDigits; i += blockDim.x) sHist[i] = 0;
    __syncthreads();
    const uint32_t n = dCount != nullptr ? min(*dCount, cap) : cap;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const K key = keys[i];
        for (uint32_t p = 0; p < passes; ++p) atomicAdd(&sHist[p * kDigits + digit_of(key, firstBit + 8 * p)], 1u);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < passes * kDigits; i += blockDim.x)
        if (sHist[i] != 0) atomicAdd(&hist[i], sHist[i]);
}

template <typename K, bool kValues, typename W, uint32_t kItems, bool kChained>
__global__ void __launch_bounds__(kSortThreads, kValues ? 3 : 4)
onesweep_kernel(const K* __restrict__ kin, K* __restrict__ kout, const uint32_t* __restrict__ vin,
                uint32_t* __restrict__ vout, const uint32_t* __restrict__ dCount, uint32_t cap,
                const uint32_t* __restrict__ hist, W* __restrict__ lookback,
                uint32_t* __restrict__ ticket, uint32_t* __restrict__ err, uint32_t shift, uint32_t spinLimit) {
    chained_entry<kChained>();
    extern __shared__ __align__(16) unsigned char smem[];
    K* sKeys = reinterpret_cast<K*>(smem);
    uint32_t* sVals = reinterpret_cast<uint32_t*>(smem + sizeof(K) * (kItems * kSortThreads));
    __shared__ uint32_t sWarpHist[kSortWarps][kDigits];
    __shared__ uint32_t sBlockStart[kDigits];
    __shared__ uint32_t sGlobal[kDigits];
    __shared__ uint32_t sScan[kSortWarps];
    __shared__ uint32_t sPart;

    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u, warp = tid >> 5;
    if (tid == 0) sPart = atomicAdd(ticket, 1u);
    for (uint32_t i = tid; i < kSortWarps * kDigits; i += kSortThreads) (&sWarpHist[0][0])[i] = 0;
    __syncthreads();
    const uint32_t n = dCount != nullptr ? min(*dCount, cap) : cap;
    const uint32_t part = sPart;
    const uint32_t base = part * (kItems * kSortThreads);
    if (base >= n) return;

    // Warp-striped load: item j of lane l is key base + 384 warp + 32 j + l.
    K key[kItems];
    uint32_t val[kItems];
    uint32_t dig[kItems];
    const uint32_t wbase = base + warp * (kItems * 32);
#pragma unroll
    for (uint32_t j = 0; j < kItems; ++j) {
        const uint32_t idx = wbase + j * 32 + lane;
        const bool ok = idx < n;
        // Past the end (only in the last partition): all-ones keys, digit
        // 255 in every pass. They rank after every real key (the ranking is
        // stable and they come last), so they take the block's last places,
        // which the write-out never reaches; their count only inflates the
        // last partition's own digit-255 total, which no partition reads.
        key[j] = ok ? kin[idx] : ~K(0);
        if (kValues) val[j] = ok ? vin[idx] : 0u;
        dig[j] = digit_of(key[j], shift);
    }

    // Stable rank inside the warp: peers with equal digits, lower lanes first;
    // items in order. Each item's group leader adds the group's size to the
    // warp's digit counter with a shared-memory atomic and passes the old
    // count to its peers. A warp's atomics on one address take effect in
    // issue order, so the items need no barrier between them: in groups of
    // kRankGroup items, every item's peer mask is found first, then every
    // leader's atomic is issued (their latencies overlap), then the old
    // counts are passed on.
    uint32_t rank[kItems];
    const uint32_t lowerLanes = (1u << lane) - 1u;
    constexpr uint32_t kRankGroup = 4;
    static_assert(kItems % kRankGroup == 0, "the rank groups must cover the items exactly");
#pragma unroll
    for (uint32_t j0 = 0; j0 < kItems; j0 += kRankGroup) {
        uint32_t peers[kRankGroup];
#pragma unroll
        for (uint32_t q = 0; q < kRankGroup; ++q) peers[q] = match_digit(dig[j0 + q]);
#pragma unroll
        for (uint32_t q = 0; q < kRankGroup; ++q) {
            const uint32_t leader = 31u - static_cast<uint32_t>(__clz(peers[q]));
            rank[j0 + q] = 0;
            if (lane == leader)
                rank[j0 + q] = atomicAdd(&sWarpHist[warp][dig[j0 + q]], static_cast<uint32_t>(__popc(peers[q])));
        }
#pragma unroll
        for (uint32_t q = 0; q < kRankGroup; ++q) {
            const uint32_t leader = 31u - static_cast<uint32_t>(__clz(peers[q]));
            rank[j0 + q] = __shfl_sync(0xFFFFFFFFu, rank[j0 + q], static_cast<int>(leader)) +
                           static_cast<uint32_t>(__popc(peers[q] & lowerLanes));
        }
    }
    __syncthreads();

    // Per digit (thread = digit): warps' exclusive offsets and the block count.
    uint32_t count = 0;
#pragma unroll
    for (uint32_t w = 0; w < kSortWarps; ++w) {
        const uint32_t c = sWarpHist[w][tid];
        sWarpHist[w][tid] = count;
        count += c;
    }
    constexpr W kFlagAggregate = LookWord<W>::kAggregate;
    constexpr W kFlagInclusive = LookWord<W>::kInclusive;
    constexpr W kValueMask = LookWord<W>::kValue;
    cuda::atomic_ref<W, cuda::thread_scope_device> mine(lookback[static_cast<size_t>(part) * kDigits + tid]);
    if (part == 0) {
        mine.store(kFlagInclusive | static_cast<W>(count), cuda::memory_order_relaxed);
    } else {
        mine.store(kFlagAggregate | static_cast<W>(count), cuda::memory_order_relaxed);
    }
    const uint32_t blockStart = block_exclusive_scan_256(count, sScan);
    const uint32_t globalStart = block_exclusive_scan_256(hist[tid], sScan);
    sBlockStart[tid] = blockStart;

    // The look-back reads kLookWords earlier partitions' words at once (their
    // loads in flight together) and sums them in order up to the first one
    // not yet published or the first inclusive one.
    uint32_t prefix = 0;
    if (part > 0) {
        int64_t p = static_cast<int64_t>(part) - 1;
        uint32_t spins = 0;
        while (p >= 0) {
            W words[kLookWords];
#pragma unroll
            for (uint32_t q = 0; q < kLookWords; ++q) {
                words[q] = kFlagInclusive;   // before partition 0: an inclusive zero
                if (p - static_cast<int64_t>(q) >= 0) {
                    cuda::atomic_ref<W, cuda::thread_scope_device> s(
                        lookback[static_cast<size_t>(p - static_cast<int64_t>(q)) * kDigits + tid]);
                    words[q] = s.load(cuda::memory_order_relaxed);
                }
            }
            uint32_t used = 0;
            bool inclusive = false;
#pragma unroll
            for (uint32_t q = 0; q < kLookWords; ++q) {
                if (inclusive || used < q || (words[q] & ~kValueMask) == 0) continue;
                prefix += static_cast<uint32_t>(words[q] & kValueMask);
                used = q + 1;
                inclusive = (words[q] & kFlagInclusive) != 0;
            }
            if (inclusive) break;
            p -= used;
            if (used == 0) {
                if (++spins > spinLimit) {
                    atomicOr(err, kErrTimeout);
                    break;
                }
                __nanosleep(20);
            }
        }
        mine.store(kFlagInclusive | static_cast<W>(prefix + count), cuda::memory_order_relaxed);
    }
    sGlobal[tid] = globalStart + prefix - blockStart;
    __syncthreads();

    // Scatter into shared memory in digit order.
#pragma unroll
    for (uint32_t j = 0; j < kItems; ++j) {
        const uint32_t d = dig[j];
        const uint32_t at = sBlockStart[d] + sWarpHist[warp][d] + rank[j];
        sKeys[at] = key[j];
        if (kValues) sVals[at] = val[j];
    }
    __syncthreads();

    // Write out: slot i of the block goes to sGlobal[digit] + i.
    const uint32_t valid = min((kItems * kSortThreads), n - base);
    for (uint32_t i = tid; i < valid; i += kSortThreads) {
        const K k = sKeys[i];
        const uint32_t at = sGlobal[digit_of(k, shift)] + i;
        kout[at] = k;
        if (kValues) vout[at] = sVals[i];
    }
}

template <typename K, bool kValues, typename W, uint32_t kItems>
cudaError_t sort_impl(K* keys, K* keysAlt, uint32_t* vals, uint32_t* valsAlt, const uint32_t* dCount,
                      uint32_t cap, uint32_t firstBit, uint32_t bits, void* scratch, uint32_t* err,
                      bool* resultInAlt, cudaStream_t stream, const SortFault* fault, const uint32_t* presetHist,
                      bool scratchZeroed) {
    *resultInAlt = false;
    if (cap == 0 || bits == 0) return cudaSuccess;
    constexpr uint32_t kTile = kItems * kSortThreads;
    const uint32_t passes = (bits + 7) / 8;
    const uint32_t parts = (cap + kTile - 1) / kTile;
    char* s = static_cast<char*>(scratch);
    uint32_t* tickets = reinterpret_cast<uint32_t*>(s);                     // kMaxPasses
    uint32_t* hist = reinterpret_cast<uint32_t*>(s + 64);                   // passes x 256
    W* lookback = reinterpret_cast<W*>(s + 64 + kMaxPasses * kDigits * 4);
    const size_t bytes = sort_scratch_bytes(cap, bits);
    cudaError_t e = scratchZeroed ? cudaSuccess : launch_zero(scratch, bytes, stream);
    if (e != cudaSuccess) return e;
    const uint32_t spinLimit = fault != nullptr && fault->pollLimit != 0 ? fault->pollLimit : kSpinLimit;
    if (fault != nullptr && fault->skipFirstPartition != 0) {
        // The last pass's tickets start at 1. Only the last pass: its input is
        // whole, so a missing prefix only moves keys to earlier slots, never
        // past the end; no later pass reads what it leaves undefined.
        e = cudaMemsetAsync(tickets + (passes - 1), 1, 1, stream);
        if (e != cudaSuccess) return e;
    }
    const uint32_t* digitCounts = hist;
    if (presetHist != nullptr) {
        digitCounts = presetHist;
    } else {
        const uint32_t histBlocks = std::max(1u, std::min(parts, 148u * 4u));
        histogram_kernel<K><<<histBlocks, kHistThreads, 0, stream>>>(keys, dCount, cap, firstBit, passes, hist);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    const size_t smem = sizeof(K) * kTile + (kValues ? sizeof(uint32_t) * kTile : 0);
    for (auto kernel : {onesweep_kernel<K, kValues, W, kItems, true>, onesweep_kernel<K, kValues, W, kItems, false>}) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    K* src = keys;
    K* dst = keysAlt;
    uint32_t* vsrc = vals;
    uint32_t* vdst = valsAlt;
    for (uint32_t p = 0; p < passes; ++p) {
        e = launch_chained(onesweep_kernel<K, kValues, W, kItems, true>, onesweep_kernel<K, kValues, W, kItems, false>, dim3(parts), dim3(kSortThreads), smem, stream,
                           static_cast<const K*>(src), dst, static_cast<const uint32_t*>(vsrc), vdst, dCount, cap,
                           digitCounts + p * kDigits, lookback + static_cast<size_t>(p) * parts * kDigits,
                           tickets + p, err, firstBit + 8 * p, spinLimit);
        if (e != cudaSuccess) return e;
        std::swap(src, dst);
        std::swap(vsrc, vdst);
    }
    *resultInAlt = (passes & 1u) != 0;
    return cudaSuccess;
}

}  // namespace

size_t sort_scratch_bytes(uint32_t cap, uint32_t bits) {
    const size_t passes = (bits + 7) / 8;
    const size_t tile = cap > kLargeKeys ? kLargeTile : kSortTile;
    const size_t parts = (static_cast<size_t>(cap) + tile - 1) / tile;
    const size_t word = 8;   // room for either word size (the 64-bit form can be asked for at any size)
    return 64 + kMaxPasses * kDigits * 4 + std::max<size_t>(passes, 1) * std::max<size_t>(parts, 1) * kDigits * word;
}

template <typename K, bool kValues>
cudaError_t sort_dispatch(K* keys, K* keysAlt, uint32_t* vals, uint32_t* valsAlt, const uint32_t* dCount,
                          uint32_t cap, uint32_t firstBit, uint32_t bits, void* scratch, uint32_t* err,
                          bool* resultInAlt, cudaStream_t stream, const SortFault* fault,
                          const uint32_t* presetHist, bool scratchZeroed) {
    const bool wide = cap > kSmallSortMax || (fault != nullptr && fault->wideWords != 0);
    const bool large = cap > kLargeKeys;
    if (!wide && !large)
        return sort_impl<K, kValues, uint32_t, kSortItems>(keys, keysAlt, vals, valsAlt, dCount, cap, firstBit, bits,
                                                           scratch, err, resultInAlt, stream, fault, presetHist, scratchZeroed);
    if (!wide)
        return sort_impl<K, kValues, uint32_t, kLargeItems>(keys, keysAlt, vals, valsAlt, dCount, cap, firstBit, bits,
                                                            scratch, err, resultInAlt, stream, fault, presetHist, scratchZeroed);
    if (!large)
        return sort_impl<K, kValues, unsigned long long, kSortItems>(keys, keysAlt, vals, valsAlt, dCount, cap,
                                                                     firstBit, bits, scratch, err, resultInAlt, stream,
                                                                     fault, presetHist, scratchZeroed);
    return sort_impl<K, kValues, unsigned long long, kLargeItems>(keys, keysAlt, vals, valsAlt, dCount, cap, firstBit,
                                                                  bits, scratch, err, resultInAlt, stream, fault, presetHist, scratchZeroed);
}

cudaError_t launch_sort_u64(uint64_t* keys, uint64_t* keysAlt, uint32_t* vals, uint32_t* valsAlt,
                            const uint32_t* dCount, uint32_t cap, uint32_t firstBit, uint32_t bits,
                            void* scratch, uint32_t* err, bool* resultInAlt, cudaStream_t stream,
                            const SortFault* fault, const uint32_t* presetHist, bool scratchZeroed) {
    if (bits > 64 || firstBit + bits > 64 || (bits + 7) / 8 > kMaxPasses) return cudaErrorInvalidValue;
    if (vals != nullptr)
        return sort_dispatch<uint64_t, true>(keys, keysAlt, vals, valsAlt, dCount, cap, firstBit, bits, scratch, err,
                                         resultInAlt, stream, fault, presetHist, scratchZeroed);
    return sort_dispatch<uint64_t, false>(keys, keysAlt, nullptr, nullptr, dCount, cap, firstBit, bits, scratch, err,
                                      resultInAlt, stream, fault, presetHist, scratchZeroed);
}

cudaError_t launch_sort_u32(uint32_t* keys, uint32_t* keysAlt, uint32_t* vals, uint32_t* valsAlt,
                            const uint32_t* dCount, uint32_t cap, uint32_t firstBit, uint32_t bits,
                            void* scratch, uint32_t* err, bool* resultInAlt, cudaStream_t stream,
                            const SortFault* fault, const uint32_t* presetHist, bool scratchZeroed) {
    if (bits > 32 || firstBit + bits > 32) return cudaErrorInvalidValue;
    if (vals != nullptr)
        return sort_dispatch<uint32_t, true>(keys, keysAlt, vals, valsAlt, dCount, cap, firstBit, bits, scratch, err,
                                         resultInAlt, stream, fault, presetHist, scratchZeroed);
    return sort_dispatch<uint32_t, false>(keys, keysAlt, nullptr, nullptr, dCount, cap, firstBit, bits, scratch, err,
                                      resultInAlt, stream, fault, presetHist, scratchZeroed);
}

}  // namespace lrt
