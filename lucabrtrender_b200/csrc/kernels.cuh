// Host-side launchers of the rasteriser's kernels (one .cu file per stage).
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/lrt_raster.h"

namespace lrt {

struct FrameParams;
struct BlendParams;
struct ProjRecord;
struct ViewParams;

// Projection fused with the touched counts, their prefix and the pair words.
// counters: [0] visible (added to), [1] pairs (written by the frame's last
// partition), [2] error bits. status: one zeroed word per 256-splat partition
// of the frame; ticket: a zeroed counter per launch; partitionBase: this
// launch's first partition in the frame; lastPartition: the frame's last.
uint32_t project_partitions(uint32_t count);
size_t project_status_bytes(uint32_t partitions);
cudaError_t launch_project_emit(const FrameParams& f, const float4* positions, const uint4* shape, const uint32_t* sh,
                                ProjRecord* proj, uint4* rects, uint32_t* touched, uint32_t* keys, uint32_t* counters,
                                uint64_t* status, uint32_t* ticket, uint32_t partitionBase, uint32_t lastPartition,
                                uint32_t slotBits, uint64_t* pairs, uint32_t capacity, cudaStream_t stream,
                                const FrameParams* fDev = nullptr, const float* filter3d = nullptr);

// The same for the differentiable parameters (means float3, log-scales
// float3, quaternions w x y z, opacity logits, SH fp16 [16][3]); also writes
// each slot's first pair index and each pair's emit index into `values`.
// Point instances as opaque discs, into the same records and pair stream.
cudaError_t launch_project_points(const FrameParams& f, const float4* positions, const uint32_t* colours,
                                  const lrt_point_style& style, ProjRecord* proj, uint4* rects, uint32_t* touched,
                                  uint32_t* keys, uint32_t* counters, uint64_t* status, uint32_t* ticket,
                                  uint32_t partitionBase, uint32_t lastPartition, uint32_t slotBits, uint64_t* pairs,
                                  uint32_t capacity, cudaStream_t stream);
cudaError_t launch_project_emit_train(const FrameParams& f, const float* means, const float* logScales,
                                      const float* quats, const float* logits, const uint16_t* sh, ProjRecord* proj,
                                      uint4* rects, uint32_t* touched, uint32_t* keys, uint32_t* offsets,
                                      uint32_t* counters, uint64_t* status, uint32_t* ticket, uint32_t partitionBase,
                                      uint32_t lastPartition, uint32_t lowBits, uint64_t* pairs, uint32_t* values,
                                      uint32_t* emitSlot, uint32_t capacity, cudaStream_t stream,
                                      const FrameParams* fDev = nullptr);

// The reference's two-sort order in two steps around a depth sort: the
// projection alone (records, rects, touched counts, depth keys; per slot the
// depth word depthKey << 32 | slot and the aux word emit_sorted reads), then,
// over the depth words sorted on bits 32-55, the pairs emitted in depth order
// as tile << 32 | slot (counters[1]: their total; status and ticket as for
// the projection, over project_partitions(n) partitions).
cudaError_t launch_project_only(const FrameParams& f, const float4* positions, const uint4* shape, const uint32_t* sh,
                                const float* filter3d, ProjRecord* proj, uint4* rects, uint32_t* touched,
                                uint32_t* keys, uint32_t* counters, uint32_t* ticket, uint64_t* aux,
                                uint64_t* depthWords, uint32_t* depthDigits,
                                uint2* rowTable, uint32_t rowCap, cudaStream_t stream);
cudaError_t launch_project_points_only(const FrameParams& f, const float4* positions, const uint32_t* colours,
                                       const lrt_point_style& style, ProjRecord* proj, uint4* rects, uint32_t* touched,
                                       uint32_t* keys, uint32_t* counters, uint32_t* ticket, uint64_t* aux,
                                       uint64_t* depthWords, uint32_t* depthDigits,
                                uint2* rowTable, uint32_t rowCap, cudaStream_t stream);
// rowTable (rowCap entries; counters[3] counts the entries asked for): each
// large splat's rows (first column, count), kept by the projection for the
// pair writes; null: none kept.
// The pairs in depth order from the depth-sorted slot words: each slot's
// first pair into offsets[slot] (the total into counters[1]), then the pair
// words tile << 32 | slot. Training frames: the emit index as the word's low
// field with emitSlot[index] = slot, or as values[] beside a slot (both null:
// not a training frame).
// tileDigits (tilePasses x 256, tilePasses 1 or 2): the tile sort's digit
// counts of the pairs written, added up there for the sort.
cudaError_t launch_emit_sorted(const uint64_t* sortedWords, uint32_t n, const ProjRecord* proj, const uint4* rects,
                               const uint32_t* touched, const uint64_t* aux, uint32_t width, uint32_t height,
                               uint32_t tilesX, uint32_t* counters, uint64_t* status, uint32_t* ticket,
                               uint32_t* offsets, uint64_t* pairs, uint32_t capacity, uint32_t* tileDigits,
                               uint32_t tilePasses, const uint2* rowTable, cudaStream_t stream,
                               uint32_t* values = nullptr, uint32_t* emitSlot = nullptr);
cudaError_t launch_project_only_train(const FrameParams& f, const float* means, const float* logScales,
                                      const float* quats, const float* logits, const uint16_t* sh, ProjRecord* proj,
                                      uint4* rects, uint32_t* touched, uint32_t* keys, uint32_t* counters,
                                      uint32_t* ticket, uint64_t* aux, uint64_t* depthWords, uint32_t* depthDigits,
                                uint2* rowTable, uint32_t rowCap, cudaStream_t stream);

size_t scan_scratch_bytes(uint32_t n);
cudaError_t launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t* total, uint32_t n, void* scratch,
                                  uint32_t* err, cudaStream_t stream);

// A planted look-back fault, for the test of the bounded waits: the last
// pass's ticket counter starts at 1, so its partition 0 is never taken and
// never publishes its counts; the partition after it polls at most
// `pollLimit` times, gives up, sets kErrTimeout and carries on (the sort's
// output is then undefined, every write still in bounds).
// `wideWords` makes a sort of fewer than 2^30 keys use the 64-bit look-back
// words that larger sorts need, so that tests can check that form.
struct SortFault {
    uint32_t skipFirstPartition = 0;
    uint32_t pollLimit = 0;   // 0: the normal limit
    uint32_t wideWords = 0;
};

size_t sort_scratch_bytes(uint32_t cap, uint32_t bits);
// presetHist: the digit counts of every pass (256 a pass, from firstBit up),
// already counted by the kernel that wrote the keys; the sort then skips its
// own counting pass over the keys. scratchZeroed: the caller has zeroed the
// sort_scratch_bytes(cap, bits) bytes of scratch on the stream already.
cudaError_t launch_sort_u64(uint64_t* keys, uint64_t* keysAlt, uint32_t* vals, uint32_t* valsAlt,
                            const uint32_t* dCount, uint32_t cap, uint32_t firstBit, uint32_t bits, void* scratch,
                            uint32_t* err, bool* resultInAlt, cudaStream_t stream, const SortFault* fault = nullptr,
                            const uint32_t* presetHist = nullptr, bool scratchZeroed = false);
cudaError_t launch_sort_u32(uint32_t* keys, uint32_t* keysAlt, uint32_t* vals, uint32_t* valsAlt,
                            const uint32_t* dCount, uint32_t cap, uint32_t firstBit, uint32_t bits, void* scratch,
                            uint32_t* err, bool* resultInAlt, cudaStream_t stream, const SortFault* fault = nullptr,
                            const uint32_t* presetHist = nullptr, bool scratchZeroed = false);

// rangesZeroed: the caller has zeroed the `tiles` ranges on the stream already.
cudaError_t launch_ranges(const uint64_t* pairs, const uint32_t* dCount, uint32_t cap, uint32_t tileShift,
                          uint2* ranges, uint32_t tiles, cudaStream_t stream, bool rangesZeroed = false);

// `bytes` (a multiple of 4, from a 4-byte aligned `p`) set to zero by a
// kernel. The frame path clears its scratch this way rather than by
// cudaMemsetAsync, which the driver may hand to a copy engine, where it
// would queue behind a caller's device-to-host copies.
cudaError_t launch_zero(void* p, size_t bytes, cudaStream_t stream);
// Up to kZeroRegions such regions in one launch.
struct ZeroRegion {
    void* p;
    size_t bytes;
};
constexpr uint32_t kZeroRegions = 6;
cudaError_t launch_zero_regions(const ZeroRegion* regions, uint32_t count, cudaStream_t stream);

// The frame's four counters stored into pinned host memory by a kernel
// (`hostMapped` is the device's address of that memory), not by a copy: a
// device-to-host copy queues behind whatever the copy engine already holds,
// such as a caller's readback of the previous image, and the frame's stream
// would wait for it.
cudaError_t launch_publish_counters(const uint32_t* counters, uint32_t* hostMapped, cudaStream_t stream);

// The frame's tiles busiest first (by buckets of log2 of their pair counts),
// the order the blends below launch them in when given one; scratch holds
// tile_order_scratch_bytes(tiles).
size_t tile_order_scratch_bytes(uint32_t tiles);
cudaError_t launch_tile_order(const uint2* ranges, uint32_t tiles, uint32_t* order, uint32_t* scratch,
                              cudaStream_t stream, const uint32_t* work = nullptr);
// The same for a training frame's backward blend, by the pairs up to each
// tile's last contributor (from the forward's per-pixel last indices);
// `work` holds a word per tile.
cudaError_t launch_tile_backward_order(const uint2* ranges, const uint32_t* pixLast, uint32_t width, uint32_t height,
                                       uint32_t tilesX, uint32_t tiles, uint32_t* order, uint32_t* scratch,
                                       uint32_t* work, cudaStream_t stream);
cudaError_t launch_blend(const BlendParams& bp, const uint2* ranges, const uint64_t* pairs, const ProjRecord* proj,
                         float4* colour, float* depth, uint32_t* err, cudaStream_t stream,
                         const uint32_t* order = nullptr);

// The views' tiles in one persistent launch; `queue` is a zeroed counter and
// `blocks` the grid size (a multiple of the SM count).
// The composite blend: disc records end a pixel's walk, and so does an under
// layer (underColour may be null: discs only).
cudaError_t launch_blend_composite(const BlendParams& bp, const uint2* ranges, const uint64_t* pairs,
                                  const ProjRecord* proj, float4* colour, float* depth, const float4* underColour,
                                  const float* underDepth, uint32_t* err, cudaStream_t stream);
cudaError_t launch_blend_batch(const BlendParams& bp, const ViewParams* views, uint32_t viewCount, const uint2* ranges,
                               const uint64_t* pairs, const ProjRecord* proj, uint32_t totalTiles, uint32_t* queue,
                               uint32_t* err, uint32_t blocks, cudaStream_t stream);
// A training batch: blend_kernel<true> per (view, tile) item, and the backward
// per item (views carry pixState, pixLast and gradColour; emit: the sorted
// pairs' emit indices).
cudaError_t launch_blend_batch_train(const BlendParams& bp, const ViewParams* views, uint32_t viewCount,
                                     const uint2* ranges, const uint64_t* pairs, const ProjRecord* proj,
                                     uint32_t totalTiles, uint32_t* queue, uint32_t* err, uint32_t blocks,
                                     cudaStream_t stream);
cudaError_t launch_blend_backward_batch(const BlendParams& bp, const ViewParams* views, uint32_t viewCount,
                                        const uint2* ranges, const uint64_t* pairs, const uint32_t* emit,
                                        const ProjRecord* proj, uint32_t totalTiles, float* partials,
                                        cudaStream_t stream);
// Training frames: `emitSlot` (when not null) maps a pair word's low field,
// the pair's emit index, to its slot; otherwise the low field is the slot and
// `emit` holds each sorted pair's emit index.
cudaError_t launch_blend_train(const BlendParams& bp, const uint2* ranges, const uint64_t* pairs,
                               const uint32_t* emitSlot, const ProjRecord* proj, float4* colour, float* depth,
                               float4* pixState, uint32_t* pixLast, uint32_t* err, cudaStream_t stream,
                               const uint32_t* order = nullptr);
cudaError_t launch_blend_backward(const BlendParams& bp, const uint2* ranges, const uint64_t* pairs,
                                  const uint32_t* emit, const uint32_t* emitSlot, const ProjRecord* proj,
                                  const float4* pixState, const uint32_t* pixLast, const float4* gradColour,
                                  float* partials, cudaStream_t stream, const uint32_t* order = nullptr);

cudaError_t launch_splat_backward(const FrameParams& f, const float* means, const float* logScales, const float* quats,
                                  const float* logits, const uint16_t* sh, const uint32_t* touched,
                                  const uint32_t* offsets, const float* partials, uint32_t partialPairs,
                                  float* gMeans, float* gLogScales, float* gQuats, float* gLogits, float* gSh,
                                  cudaStream_t stream);
// The same over a chunk of up to 16 views (FrameParams in device memory,
// touched and offsets one array of `count` per view), adding the views'
// gradients in view order and writing each buffer once; accumulate: add to
// what the buffers hold.
cudaError_t launch_splat_backward_views(const FrameParams* framesDev, uint32_t views, uint32_t count,
                                        const float* means, const float* logScales, const float* quats,
                                        const float* logits, const uint16_t* sh, const uint32_t* touched,
                                        const uint32_t* offsets, const float* partials, uint32_t partialPairs,
                                        float* gMeans, float* gLogScales, float* gQuats, float* gLogits, float* gSh,
                                        bool accumulate, cudaStream_t stream);

cudaError_t launch_math_eval(int fn, const float* x, float* y, uint32_t n, cudaStream_t stream);

// Cloud decode (decode.cu): validate, compact and pack in one kernel.
// scratch: decode_status_bytes(count) bytes, zeroed; err: the status word.
size_t decode_status_bytes(uint32_t count);
cudaError_t launch_decode_splats(const float* raw, uint32_t count, const lrt_splat_encoding& e, uint32_t keep,
                                 uint32_t shWords, float4* positions, uint4* shape, uint32_t* sh, void* scratch,
                                 uint32_t* err, cudaStream_t stream);
cudaError_t launch_decode_points(const float* raw, uint32_t count, uint32_t colourKind, float detail,
                                 float4* positions, uint32_t* colours, void* scratch, uint32_t* err,
                                 cudaStream_t stream);

// Parity metrics (compare.cu).
cudaError_t launch_compare_images(const float4* a, const float4* b, uint32_t pixels, uint32_t* histogram,
                                  cudaStream_t stream);
cudaError_t launch_compare_hdr(const float4* a, const float4* b, uint32_t width, uint32_t height, uint32_t* histogram,
                               float* rowError, float* total, cudaStream_t stream);
cudaError_t launch_count_different(const uint32_t* a, const uint32_t* b, uint32_t count, uint64_t* total,
                                   cudaStream_t stream);

// The L1 training loss (loss.cu).
size_t l1_scratch_bytes();
cudaError_t launch_l1_loss(const float4* colour, const float* target, uint32_t pixels, float* scratch, float* loss,
                           cudaStream_t stream);
cudaError_t launch_l1_grad(const float4* colour, const float* target, uint32_t pixels, const float* gradLoss,
                           float4* gradColour, cudaStream_t stream);


// Levels of detail (lod.cu).
constexpr uint32_t kLodLevels = 10;   // 30-bit Morton codes, lod_common.slang:36
constexpr uint32_t kLodMomentsHead = 13;   // lod_common.slang:38-40

// What the build keeps on the device between its kernels: the bounds, the
// cubic extent, the splat count the sort reads, and per level the number of
// splats that begin a group there and at no coarser level (index = level;
// kLodLevels + 1 counts splats whose codes equal their predecessor's).
struct LodGlobals {
    float lo[3], hi[3], extent;
    uint32_t count;
    uint32_t firstLevel[kLodLevels + 2];
    uint32_t groupTotals[kLodLevels + 1];   // per level: the groups its compaction found
    uint32_t pad[3];
};

// One instance's cut: the cloud's layout and this view's test.
struct LodCutParams {
    uint32_t merged, count, levels, coarsest;   // coarsest: octree level of stored level 0
    uint32_t levelBase[kLodLevels + 2];         // first merged Gaussian of each stored level; [levels] = merged
    uint32_t shWords, capacity, ortho, pad0;
    float lo[3], extent;
    float eye[3], pixelsPerUnit;
    float threshold, pad1, pad2, pad3;
};

struct LodSplatArrays {
    float4* positions;
    uint4* shape;
    uint32_t* sh;
};

cudaError_t launch_lod_bounds(const float4* positions, uint32_t count, const float* given, LodGlobals* globals,
                              float* partial, cudaStream_t stream);
size_t lod_bounds_partial_bytes();
cudaError_t launch_lod_morton(const float4* positions, uint32_t count, const LodGlobals* globals, uint32_t* keys,
                              uint32_t* order, cudaStream_t stream);
cudaError_t launch_lod_reorder(const uint32_t* order, const uint32_t* codes, uint32_t count, uint32_t shWords,
                               const float4* srcPositions, const uint4* srcShape, const uint32_t* srcSh,
                               LodSplatArrays store, LodGlobals* globals, cudaStream_t stream);
// status: compaction_status_bytes(count, lod_compaction_threads()) zeroed bytes.
uint32_t lod_compaction_threads();
// capacity: the groups the output arrays hold (writes past it are dropped).
cudaError_t launch_lod_finest_groups(const uint32_t* codes, uint32_t count, uint32_t level, uint32_t capacity,
                                     uint32_t* starts, uint32_t* cells, void* status, uint32_t* total, uint32_t* err,
                                     cudaStream_t stream);
cudaError_t launch_lod_parent_groups(const uint32_t* fineCells, uint32_t fineCount, uint32_t capacity,
                                     uint32_t* cells, uint32_t* firstChild, void* status, uint32_t* total,
                                     uint32_t* err, cudaStream_t stream);
cudaError_t launch_lod_leaf_moments(const LodSplatArrays store, uint32_t count, uint32_t restPerColour,
                                    uint32_t shWords, const uint32_t* starts, uint32_t groups, float* moments,
                                    cudaStream_t stream);
cudaError_t launch_lod_merge_moments(const uint32_t* firstChild, uint32_t groups, uint32_t fineGroups,
                                     const float* fineMoments, float* moments, uint32_t stride, cudaStream_t stream);
cudaError_t launch_lod_finalize(const float* moments, uint32_t groups, uint32_t restPerColour, uint32_t shWords,
                                LodSplatArrays merged, cudaStream_t stream);
// scratch: lod_cut_scratch_bytes(merged + count) bytes (per block a bitmask
// and a count, all written by the cut); counts: two words (drawn, of which
// merged), written by the cut.
size_t lod_cut_scratch_bytes(uint32_t items);
cudaError_t launch_lod_cut(const LodCutParams& c, const uint32_t* cells, const uint32_t* codes,
                           const LodSplatArrays merged, const LodSplatArrays store, LodSplatArrays out,
                           void* scratch, uint32_t* counts, cudaStream_t stream);

}  // namespace lrt
