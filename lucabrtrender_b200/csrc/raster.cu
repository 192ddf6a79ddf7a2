// The C-ABI rasteriser: lrt_rast_create / lrt_rast_render / ... (see
// include/lrt_raster.h). Host orchestration of one frame, in the reference's
// order (modules/render/src/TileRasterizer.cpp:188-484):
//
//   project + count + emit (one kernel per instance, offsets by look-back)
//   -> onesweep sort of the pairs' (tile | depth) key bits -> tile ranges
//   -> blend -> one readback of the visible and pair counts and the status
//
// The reference reads the counts back in the middle of the frame to size the
// pair buffers; here the pairs go into a buffer sized before the frame, and a
// frame that reports more pairs than it held is drawn again with room for
// them (once per growth, so steady frames never repeat).
//
// Buffers belong to the handle and grow by 1.5x (TileRasterizer.cpp:26-32);
// targets and clouds belong to the caller. Stage times come from CUDA events
// on the caller's stream.
#include "../../include/lrt_raster.h"
#include "kernels.cuh"
#include "raster_common.cuh"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <algorithm>
#include <vector>

#include "rast_handle.h"

extern "C" {

uint32_t lrt_abi_version(void) { return LRT_ABI_VERSION; }

int lrt_rast_create(lrt_rast** out, int device) {
    if (out == nullptr) return LRT_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return LRT_DEVICE_FAILURE;
    if (device < 0 || device >= count) return LRT_INVALID_ARGUMENT;
    DeviceScope scope(device);
    lrt_rast* r = new lrt_rast();
    r->device = device;
    bool ok = cudaMallocHost(reinterpret_cast<void**>(&r->hostCounters), 64) == cudaSuccess &&
              cudaMallocHost(reinterpret_cast<void**>(&r->ringHost), lrt_rast::kRing * 16) == cudaSuccess &&
              cudaHostGetDevicePointer(reinterpret_cast<void**>(&r->hostCountersDev), r->hostCounters, 0) ==
                  cudaSuccess &&
              cudaHostGetDevicePointer(reinterpret_cast<void**>(&r->ringHostDev), r->ringHost, 0) == cudaSuccess &&
              ensure(r->counters, 64) == cudaSuccess;
    for (auto& e : r->ev) ok = ok && cudaEventCreate(&e) == cudaSuccess;
    for (auto& e : r->ringEvent) ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&r->frameDone, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        lrt_rast_destroy(r);
        cudaGetLastError();
        return LRT_DEVICE_FAILURE;
    }
    *out = r;
    return LRT_OK;
}

void lrt_rast_destroy(lrt_rast* r) {
    if (r == nullptr) return;
    DeviceScope scope(r->device);
    if (r->frameDoneSet) cudaEventSynchronize(r->frameDone);   // a backward may still read the buffers
    for (DeviceBuffer* b : {&r->proj, &r->rects, &r->touched, &r->keys, &r->pairs, &r->pairsAlt,
                            &r->ranges, &r->scanScratch, &r->sortScratch, &r->counters, &r->algoKeysAlt,
                            &r->algoValsAlt, &r->depthWords, &r->depthWordsAlt, &r->splatAux, &r->rowTable,
                            &r->pairValues, &r->pairValuesAlt, &r->pairOffsets, &r->pixState, &r->pixLast, &r->partials, &r->metricScratch, &r->lossScratch, &r->trainBatchGrad,
                            &r->trainBatchViews, &r->trainBatchLoss, &r->lodBuild.globals,
                            &r->lodBuild.partial, &r->lodBuild.keys, &r->lodBuild.keysAlt, &r->lodBuild.order,
                            &r->lodBuild.orderAlt, &r->lodBuild.sortScratch, &r->lodBuild.status,
                            &r->lodBuild.firstChild, &r->lodBuild.moments, &r->lodBuild.err})
        release(*b);
    if (r->ringTail < r->ringHead) cudaDeviceSynchronize();   // enqueued frames still write the ring
    if (r->hostCounters != nullptr) cudaFreeHost(r->hostCounters);
    if (r->ringHost != nullptr) cudaFreeHost(r->ringHost);
    if (r->metricHost != nullptr) cudaFreeHost(r->metricHost);
    for (auto& e : r->ev)
        if (e != nullptr) cudaEventDestroy(e);
    for (auto& e : r->ringEvent)
        if (e != nullptr) cudaEventDestroy(e);
    if (r->frameDone != nullptr) cudaEventDestroy(r->frameDone);
    auto& B = r->batch;
    for (DeviceBuffer* b : {&B.records, &B.ranges, &B.params, &B.counters, &B.queue}) release(*b);
    if (B.hostParams != nullptr) cudaFreeHost(B.hostParams);
    if (B.hostCounters != nullptr) cudaFreeHost(B.hostCounters);
    if (B.graph != nullptr) cudaGraphExecDestroy(B.graph);
    for (cudaEvent_t e : {B.in, B.out, B.start, B.end})
        if (e != nullptr) cudaEventDestroy(e);
    if (B.stream != nullptr) cudaStreamDestroy(B.stream);
    auto& TB = r->trainBatch;
    release(TB.counters);
    if (TB.hostParams != nullptr) cudaFreeHost(TB.hostParams);
    if (TB.hostCounters != nullptr) cudaFreeHost(TB.hostCounters);
    if (TB.graph != nullptr) cudaGraphExecDestroy(TB.graph);
    for (cudaEvent_t e : {TB.in, TB.out, TB.start, TB.end})
        if (e != nullptr) cudaEventDestroy(e);
    if (TB.stream != nullptr) cudaStreamDestroy(TB.stream);
    for (DeviceBuffer* b : {&r->filterCameras, &r->filterScratch}) release(*b);
    release_cut_frames(r);
    delete r;
}

const char* lrt_rast_last_error(const lrt_rast* r) { return r == nullptr ? "no handle" : r->error.c_str(); }

}  // extern "C"

namespace {

// One projection launch of a frame: a packed cloud instance, or the
// differentiable parameters of the training path.
// One frame, TileRasterizer.cpp:188-484 in this library's stage order. `train`
// selects the training variants (emit indices carried through the sort,
// per-slot pair offsets, per-pixel blend state for the backward pass).
// `deferred`: enqueue the frame and return without waiting (training frames
// after the first); the counts and status arrive in pinned memory and the
// backward pass checks them.
int render_frame(lrt_rast* r, const lrt_projection* pr, const std::vector<CloudDesc>& clouds,
                 const lrt_render_settings* s, lrt_targets* targets, lrt_frame_stats* stats, void* streamPtr,
                 bool train, std::chrono::steady_clock::time_point frameStart, bool deferred = false,
                 const lrt_targets* under = nullptr, bool composite = false) {
    if (s->width == 0 || s->height == 0) return fail(r, LRT_INVALID_ARGUMENT, "a frame needs a size");
    if (s->width > lrt::kMaxFrameSide || s->height > lrt::kMaxFrameSide)
        return fail(r, LRT_UNSUPPORTED, "a frame side above 2^19 pixels");
    const lrt::ChainScope chain(uint64_t{s->width} * s->height >= lrt::kChainMinPixels);
    if (targets->width != s->width || targets->height != s->height || targets->colour == nullptr ||
        targets->depth == nullptr)
        return fail(r, LRT_INVALID_ARGUMENT, "the targets are not the frame's size");
    uint64_t total = 0;
    uint64_t partitions = 0;
    for (const CloudDesc& c : clouds) {
        total += c.count;
        partitions += lrt::project_partitions(c.count);
    }
    const uint32_t launches = static_cast<uint32_t>(clouds.size());
    if (total > 0xFFFFFFFFull) return fail(r, LRT_UNSUPPORTED, "more than 2^32 splats in one frame");
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    // The handle's buffers serve one frame at a time: a frame on another
    // stream than the last one waits for it.
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    const uint32_t slots = static_cast<uint32_t>(total);
    const uint32_t tilesX = (s->width + lrt::kTile - 1) / lrt::kTile;
    const uint32_t tilesY = (s->height + lrt::kTile - 1) / lrt::kTile;
    const uint32_t tiles = tilesX * tilesY;
    const uint32_t tileBits = bits_for(tiles);
    // A frame takes the reference's two sorts: the projection alone, a sort
    // of the slots' depth words, the pairs emitted in depth order as
    // tile << 32 | slot (or emit index), and a stable sort of those on the tile
    // bits (TileRasterizer.cpp:401-457).

    // Buffers (TileRasterizer.cpp:105-177).
    if (slots > r->splatCap) {
        const uint32_t cap = grow(r->splatCap, slots);
        LRT_CUDA(r, ensure(r->proj, size_t{cap} * sizeof(ProjRecord)), "splat records");
        LRT_CUDA(r, ensure(r->rects, size_t{cap} * 16), "tile rects");
        LRT_CUDA(r, ensure(r->touched, size_t{cap} * 4), "touched counts");
        LRT_CUDA(r, ensure(r->keys, size_t{cap} * 4), "depth keys");
        r->splatCap = cap;
    }
    LRT_CUDA(r, ensure(r->depthWords, size_t{r->splatCap} * 8), "depth words");
    LRT_CUDA(r, ensure(r->depthWordsAlt, size_t{r->splatCap} * 8), "depth words");
    LRT_CUDA(r, ensure(r->splatAux, size_t{r->splatCap} * 16), "tile masks");
    // The row table: one entry a slot to start with, grown to what a frame
    // asked for (a splat past its end is planned again when written).
    if (r->rowCap == 0) r->rowCap = std::max<uint32_t>(r->splatCap, 1024);
    LRT_CUDA(r, ensure(r->rowTable, size_t{r->rowCap} * sizeof(uint2)), "row table");
    LRT_CUDA(r, ensure(r->pairOffsets, size_t{std::max(slots, 1u)} * 4), "pair offsets");
    if (train) {
        LRT_CUDA(r, ensure(r->pixState, size_t{s->width} * s->height * 16), "pixel state");
        LRT_CUDA(r, ensure(r->pixLast, size_t{s->width} * s->height * 4), "pixel state");
    }
    // Look-back status words and a ticket per projection launch, plus one
    // for the emission over the frame's slots in depth order; then the two
    // sorts' digit counts (3 passes of the depth sort, up to 2 of the tile
    // sort), counted by the kernels that write the keys.
    const size_t ticketsEnd = lrt::project_status_bytes(static_cast<uint32_t>(partitions)) + size_t{launches + 1} * 4;
    const size_t digitsAt = (ticketsEnd + 15) & ~size_t{15};
    const size_t statusBytes = digitsAt + 5 * 256 * 4;
    LRT_CUDA(r, ensure(r->scanScratch, std::max<size_t>(statusBytes, 16)), "projection scratch");
    if (tiles > r->tileCap) {
        LRT_CUDA(r, ensure(r->ranges, size_t{tiles} * 8), "tile ranges");
        // order, its scratch, and the backward's per-tile work
        LRT_CUDA(r, ensure(r->tileOrder, size_t{tiles} * 8 + lrt::tile_order_scratch_bytes(tiles)), "tile order");
        r->tileCap = tiles;
    }
    // Pairs are emitted on the device into a buffer of the capacity known
    // before the frame; a frame that emits more is drawn again once, with the
    // buffers grown to the count it reported.
    if (r->pairCap == 0)
        r->pairCap = std::max<uint32_t>(1024, static_cast<uint32_t>(std::min<uint64_t>(uint64_t{slots} * 4, 0xFFFFFFFFull)));
    uint32_t* counters = static_cast<uint32_t*>(r->counters.ptr);
    uint32_t* err = counters + 2;
    uint64_t* status = static_cast<uint64_t*>(r->scanScratch.ptr);
    uint32_t* tickets = reinterpret_cast<uint32_t*>(static_cast<char*>(r->scanScratch.ptr) +
                                                    lrt::project_status_bytes(static_cast<uint32_t>(partitions)));
    uint32_t* depthDigits = reinterpret_cast<uint32_t*>(static_cast<char*>(r->scanScratch.ptr) + digitsAt);
    uint32_t* tileDigits = depthDigits + 3 * 256;
    const uint32_t tilePasses = (tileBits + 7) / 8 <= 2 ? (tileBits + 7) / 8 : 0u;
    const uint32_t lastPartition = partitions > 0 ? static_cast<uint32_t>(partitions - 1) : 0u;
    uint32_t visible = 0, pairs = 0, statusBits = 0;
    const uint64_t* sorted = nullptr;
    const uint32_t* sortedValues = nullptr;
    BlendParams bp{};
    bp.width = s->width;
    bp.height = s->height;
    bp.tilesX = tilesX;
    bp.tilesY = tilesY;
    bp.depthMode = s->depth_mode;
    bp.linearise = s->linearise ? 1u : 0u;
    bp.depthThreshold = s->depth_threshold;
    for (int a = 0; a < 4; ++a) bp.bg[a] = s->background[a];
    FrameParams lastParams{};
    // Training frames carry each pair's emit index to the backward pass: the
    // pair word's low field (with an emit index -> slot map for the blend),
    // or, when asked for, a sort value beside a word whose low field is the
    // slot. Other frames' words hold the slot.
    const bool valuesAsked = train && !clouds.empty() && clouds[0].train != nullptr &&
                             (clouds[0].train->flags & LRT_TRAIN_SORT_VALUES) != 0;
    const bool lowIsEmit = train && !valuesAsked;
    bp.slotBits = 32;
    bp.tileShift = 32;
    for (int attempt = 0; attempt < 2; ++attempt) {
        LRT_CUDA(r, ensure(r->pairs, size_t{r->pairCap} * 8), "pairs");
        LRT_CUDA(r, ensure(r->pairsAlt, size_t{r->pairCap} * 8), "pairs");
        if (train) {
            LRT_CUDA(r, ensure(r->pairValues, size_t{r->pairCap} * 4), "pair values");
            if (!lowIsEmit) LRT_CUDA(r, ensure(r->pairValuesAlt, size_t{r->pairCap} * 4), "pair values");
        }
        // The two sorts' scratch side by side, so that one launch clears it
        // with the counters, the projection's scratch and the tile ranges.
        const size_t depthScratch = lrt::sort_scratch_bytes(slots, 24);
        const size_t tileScratchAt = (depthScratch + 255) & ~size_t{255};
        const size_t tileScratch = lrt::sort_scratch_bytes(r->pairCap, tileBits);
        LRT_CUDA(r, ensure(r->sortScratch, tileScratchAt + tileScratch), "sort scratch");
        void* tileSortScratch = static_cast<char*>(r->sortScratch.ptr) + tileScratchAt;
        const lrt::ZeroRegion clear[] = {{counters, 16},
                                         {r->scanScratch.ptr, statusBytes},
                                         {r->sortScratch.ptr, depthScratch},
                                         {tileSortScratch, tileScratch},
                                         {r->ranges.ptr, size_t{tiles} * sizeof(uint2)}};
        LRT_CUDA(r, lrt::launch_zero_regions(clear, 5, stream), "frame scratch");
        uint64_t* pairBuf = static_cast<uint64_t*>(r->pairs.ptr);
        uint32_t* valueBuf = train && !lowIsEmit ? static_cast<uint32_t*>(r->pairValues.ptr) : nullptr;
        uint32_t* emitSlot = train && lowIsEmit ? static_cast<uint32_t*>(r->pairValues.ptr) : nullptr;

        // --- project, count -------------------------------------------------------
        LRT_CUDA(r, cudaEventRecord(r->ev[0], stream), "event");
        uint32_t base = 0, launch = 0;
        uint64_t* depthWords = static_cast<uint64_t*>(r->depthWords.ptr);
        uint64_t* aux = static_cast<uint64_t*>(r->splatAux.ptr);
        for (const CloudDesc& c : clouds) {
            const FrameParams f = frame_params(pr, s, c, tilesX, tilesY, base);
            lastParams = f;
            if (c.point != nullptr) {
                const lrt_gpu_points& g = *c.point->points;
                LRT_CUDA(r,
                         lrt::launch_project_points_only(
                             f, static_cast<const float4*>(g.positions), static_cast<const uint32_t*>(g.colours),
                             c.point->style, static_cast<ProjRecord*>(r->proj.ptr), static_cast<uint4*>(r->rects.ptr),
                             static_cast<uint32_t*>(r->touched.ptr), static_cast<uint32_t*>(r->keys.ptr), counters,
                             tickets + launch, aux, depthWords, depthDigits, static_cast<uint2*>(r->rowTable.ptr),
                             r->rowCap, stream),
                         "points");
            } else if (c.train != nullptr) {
                const lrt_train_params& t = *c.train;
                LRT_CUDA(r,
                         lrt::launch_project_only_train(
                             f, static_cast<const float*>(t.means), static_cast<const float*>(t.log_scales),
                             static_cast<const float*>(t.quats), static_cast<const float*>(t.opacity_logits),
                             static_cast<const uint16_t*>(t.sh), static_cast<ProjRecord*>(r->proj.ptr),
                             static_cast<uint4*>(r->rects.ptr), static_cast<uint32_t*>(r->touched.ptr),
                             static_cast<uint32_t*>(r->keys.ptr), counters, tickets + launch, aux, depthWords,
                             depthDigits, static_cast<uint2*>(r->rowTable.ptr), r->rowCap, stream),
                         "project");
            } else {
                LRT_CUDA(r,
                         lrt::launch_project_only(
                             f, static_cast<const float4*>(c.packed->positions),
                             static_cast<const uint4*>(c.packed->shape), static_cast<const uint32_t*>(c.packed->sh),
                             static_cast<const float*>(c.packed->filter3d), static_cast<ProjRecord*>(r->proj.ptr),
                             static_cast<uint4*>(r->rects.ptr), static_cast<uint32_t*>(r->touched.ptr),
                             static_cast<uint32_t*>(r->keys.ptr), counters, tickets + launch, aux, depthWords,
                             depthDigits, static_cast<uint2*>(r->rowTable.ptr), r->rowCap, stream),
                         "project");
            }
            base += c.count;
            launch += 1;
        }
        LRT_CUDA(r, cudaEventRecord(r->ev[1], stream), "event");
        // --- depth sort of the slots (24-bit keys; ties stay in slot order) ------------
        bool depthInAlt = false;
        LRT_CUDA(r,
                 lrt::launch_sort_u64(depthWords, static_cast<uint64_t*>(r->depthWordsAlt.ptr), nullptr, nullptr,
                                      nullptr, slots, 32, 24, r->sortScratch.ptr, err, &depthInAlt, stream, nullptr,
                                      depthDigits, true),
                 "depth sort");
        const uint64_t* byDepth = depthInAlt ? static_cast<const uint64_t*>(r->depthWordsAlt.ptr) : depthWords;
        LRT_CUDA(r, cudaEventRecord(r->ev[4], stream), "event");
        // --- pairs in depth order ----------------------------------------------------------
        LRT_CUDA(r,
                 lrt::launch_emit_sorted(byDepth, slots, static_cast<ProjRecord*>(r->proj.ptr),
                                         static_cast<uint4*>(r->rects.ptr), static_cast<uint32_t*>(r->touched.ptr),
                                         aux, s->width, s->height, tilesX, counters, status, tickets + launches,
                                         static_cast<uint32_t*>(r->pairOffsets.ptr), pairBuf, r->pairCap,
                                         tilePasses != 0 ? tileDigits : nullptr, tilePasses,
                                         static_cast<const uint2*>(r->rowTable.ptr), stream, valueBuf, emitSlot),
                 "emit");
        LRT_CUDA(r, cudaEventRecord(r->ev[5], stream), "event");
        // --- stable sort on the tile bits + ranges -------------------------------------------
        bool inAlt = false;
        LRT_CUDA(r,
                 lrt::launch_sort_u64(pairBuf, static_cast<uint64_t*>(r->pairsAlt.ptr), valueBuf,
                                      valueBuf != nullptr ? static_cast<uint32_t*>(r->pairValuesAlt.ptr) : nullptr,
                                      counters + 1, r->pairCap, 32, tileBits, tileSortScratch, err, &inAlt, stream,
                                      nullptr, tilePasses != 0 ? tileDigits : nullptr, true),
                 "tile sort");
        sorted = inAlt ? static_cast<uint64_t*>(r->pairsAlt.ptr) : pairBuf;
        if (valueBuf != nullptr) sortedValues = inAlt ? static_cast<uint32_t*>(r->pairValuesAlt.ptr) : valueBuf;
        LRT_CUDA(r,
                 lrt::launch_ranges(sorted, counters + 1, r->pairCap, 32, static_cast<uint2*>(r->ranges.ptr), tiles,
                                    stream, true),
                 "ranges");
        // The blend takes the tiles busiest first (the composite blend keeps
        // index order).
        uint32_t* tileOrder = composite ? nullptr : static_cast<uint32_t*>(r->tileOrder.ptr);
        if (tileOrder != nullptr)
            LRT_CUDA(r, lrt::launch_tile_order(static_cast<uint2*>(r->ranges.ptr), tiles, tileOrder, tileOrder + tiles,
                                               stream),
                     "tile order");
        LRT_CUDA(r, cudaEventRecord(r->ev[2], stream), "event");

        // --- blend ------------------------------------------------------------------
        if (train) {
            LRT_CUDA(r,
                     lrt::launch_blend_train(bp, static_cast<uint2*>(r->ranges.ptr), sorted, emitSlot,
                                             static_cast<ProjRecord*>(r->proj.ptr),
                                             static_cast<float4*>(targets->colour), static_cast<float*>(targets->depth),
                                             static_cast<float4*>(r->pixState.ptr),
                                             static_cast<uint32_t*>(r->pixLast.ptr), err, stream, tileOrder),
                     "blend");
        } else if (composite) {
            LRT_CUDA(r,
                     lrt::launch_blend_composite(
                         bp, static_cast<uint2*>(r->ranges.ptr), sorted, static_cast<ProjRecord*>(r->proj.ptr),
                         static_cast<float4*>(targets->colour), static_cast<float*>(targets->depth),
                         under != nullptr ? static_cast<const float4*>(under->colour) : nullptr,
                         under != nullptr ? static_cast<const float*>(under->depth) : nullptr, err, stream),
                     "blend");
        } else {
            LRT_CUDA(r,
                     lrt::launch_blend(bp, static_cast<uint2*>(r->ranges.ptr), sorted,
                                       static_cast<ProjRecord*>(r->proj.ptr), static_cast<float4*>(targets->colour),
                                       static_cast<float*>(targets->depth), err, stream, tileOrder),
                     "blend");
        }
        LRT_CUDA(r, cudaEventRecord(r->ev[3], stream), "event");
        const bool ring = deferred && !train;
        const uint32_t slot = static_cast<uint32_t>(r->ringHead % lrt_rast::kRing);
        LRT_CUDA(r, lrt::launch_publish_counters(counters, ring ? r->ringHostDev + 4 * slot : r->hostCountersDev, stream),
                 "readback");
        LRT_CUDA(r, cudaEventRecord(r->frameDone, stream), "event");
        r->frameDoneSet = true;
        if (ring) {
            LRT_CUDA(r, cudaEventRecord(r->ringEvent[slot], stream), "event");
            r->ringCap[slot] = r->pairCap;
            r->ringHead += 1;
        }
        if (deferred) {
            r->debug.proj = r->proj.ptr;
            r->debug.rects = r->rects.ptr;
            r->debug.touched = r->touched.ptr;
            r->debug.depth_keys = r->keys.ptr;
            r->debug.pairs = sorted;
            r->debug.ranges = r->ranges.ptr;
            r->debug.slots = slots;
            r->debug.tiles = tiles;
            r->debug.slot_bits = 32u;
            r->debug.depth_bits = 0u;
            r->debug.tile_bits = tileBits;
            r->pendingStream = stream;
            if (train) LRT_CUDA(r, cudaEventRecord(r->ev[6], stream), "event");
            if (train) {
                r->trainFrame = lastParams;
                r->trainBlend = bp;
                r->trainSorted = sorted;
                r->trainSortedValues = sortedValues;
                r->trainEmitSlot = emitSlot;
                r->trainPairs = r->pairCap;   // an upper bound until the status is read
                r->trainReady = true;
                r->trainPending = true;
            }
            if (stats != nullptr) {
                std::memset(stats, 0, sizeof(*stats));
                stats->splats = slots;
                stats->total_ms =
                    std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - frameStart).count();
            }
            return LRT_OK;
        }
        LRT_CUDA(r, cudaStreamSynchronize(stream), "frame");
        visible = r->hostCounters[0];
        pairs = r->hostCounters[1];
        statusBits = r->hostCounters[2];
        if (statusBits & lrt::kErrTooManyPairs) return fail(r, LRT_UNSUPPORTED, "more than 2^32 pairs in one frame");
        if (pairs <= r->pairCap) break;
        r->pairCap = grow(r->pairCap, pairs);   // draw again with room for every pair
        statusBits &= ~lrt::kErrOverflow;
    }
    // Rows the frame's large splats asked for beyond the row table: the next
    // frame's table holds them (this one planned those rows again).
    if (r->hostCounters[3] > r->rowCap) r->rowCap = grow(r->rowCap, r->hostCounters[3]);

    r->debug.proj = r->proj.ptr;
    r->debug.rects = r->rects.ptr;
    r->debug.touched = r->touched.ptr;
    r->debug.depth_keys = r->keys.ptr;
    r->debug.pairs = sorted;
    r->debug.ranges = r->ranges.ptr;
    r->debug.slots = slots;
    r->debug.pairs_count = pairs;
    r->debug.tiles = tiles;
    r->debug.slot_bits = 32u;
    r->debug.depth_bits = 0u;
    r->debug.tile_bits = tileBits;
    r->debug.visible = visible;
    r->trainReady = false;
    r->trainPending = false;
    if (train) {
        r->trainFrame = lastParams;
        r->trainBlend = bp;
        r->trainSorted = sorted;
        r->trainSortedValues = sortedValues;
        r->trainEmitSlot = lowIsEmit ? static_cast<uint32_t*>(r->pairValues.ptr) : nullptr;
        r->trainPairs = pairs;
        r->trainReady = true;
    }

    if (stats != nullptr) {
        std::memset(stats, 0, sizeof(*stats));
        stats->splats = slots;
        stats->visible = visible;
        stats->pairs = pairs;
        if (s->time_stages) {
            stats->project_ms = event_ms(r->ev[0], r->ev[1]);
            stats->depth_sort_ms = event_ms(r->ev[1], r->ev[4]);
            stats->emit_ms = event_ms(r->ev[4], r->ev[5]);
            stats->tile_sort_ms = event_ms(r->ev[5], r->ev[2]);
            stats->blend_ms = event_ms(r->ev[2], r->ev[3]);
        }
        stats->total_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - frameStart).count();
    }
    if (statusBits & lrt::kErrTimeout) return fail(r, LRT_TIMEOUT, "a bounded device wait gave up");
    if (statusBits & lrt::kErrOverflow || pairs > r->pairCap) return fail(r, LRT_OVERFLOW, "pair capacity exceeded");
    return LRT_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

int collect_clouds(lrt_rast* r, const lrt_splat_instance* instances, uint32_t n, std::vector<CloudDesc>& clouds) {
    for (uint32_t k = 0; k < n; ++k) {
        const lrt_gpu_splats* c = instances[k].splats;
        if (c == nullptr || c->count == 0) continue;
        if (c->positions == nullptr || c->shape == nullptr)
            return fail(r, LRT_INVALID_ARGUMENT, "a cloud without positions or shape");
        if (c->rest_per_colour > 0 && c->sh == nullptr) return fail(r, LRT_INVALID_ARGUMENT, "a cloud without harmonics");
        if (c->rest_per_colour > 0 && c->sh_words < (c->rest_per_colour * 3 + 1) / 2)
            return fail(r, LRT_INVALID_ARGUMENT, "sh_words too small for rest_per_colour");
        CloudDesc d;
        d.packed = c;
        d.objectToWorld = instances[k].object_to_world;
        d.edit = &instances[k].edit;
        d.count = c->count;
        clouds.push_back(d);
    }
    return LRT_OK;
}

uint32_t total_slots(const std::vector<CloudDesc>& clouds) {
    uint64_t total = 0;
    for (const CloudDesc& c : clouds) total += c.count;
    return static_cast<uint32_t>(std::min<uint64_t>(total, 0xFFFFFFFFull));
}

// Reads the counts of the oldest enqueued plain frame (waiting for it when
// `wait`); false when it has not finished and `wait` is not set.
bool read_oldest(lrt_rast* r, bool wait) {
    const uint32_t slot = static_cast<uint32_t>(r->ringTail % lrt_rast::kRing);
    if (wait) {
        if (cudaEventSynchronize(r->ringEvent[slot]) != cudaSuccess) return false;
    } else if (cudaEventQuery(r->ringEvent[slot]) != cudaSuccess) {
        cudaGetLastError();   // cudaErrorNotReady is not an error to keep
        return false;
    }
    const uint32_t* c = r->ringHost + 4 * slot;
    r->asyncVisible = c[0];
    r->asyncPairs = c[1];
    r->plainSeenPairs = c[1];
    if (c[1] > r->ringCap[slot] || (c[2] & lrt::kErrTooManyPairs) != 0) {
        r->asyncOverflows += 1;
        r->pairCap = std::max(r->pairCap, grow(r->pairCap, c[1]));
    }
    if (c[2] & lrt::kErrTimeout) r->asyncTimeouts += 1;
    r->debug.visible = c[0];
    r->debug.pairs_count = std::min(c[1], r->ringCap[slot]);
    r->ringTail += 1;
    return true;
}

// Waits for every enqueued plain frame and reports what they met since the
// last report: OVERFLOW (those frames' images are incomplete; the buffers are
// grown) or TIMEOUT.
int settle_async(lrt_rast* r) {
    DeviceScope scope(r->device);
    while (r->ringTail < r->ringHead) {
        if (!read_oldest(r, true)) return fail(r, LRT_DEVICE_FAILURE, "waiting for an enqueued frame failed");
    }
    const uint32_t overflows = r->asyncOverflows, timeouts = r->asyncTimeouts;
    r->asyncOverflows = 0;
    r->asyncTimeouts = 0;
    if (overflows != 0)
        return fail(r, LRT_OVERFLOW,
                    std::to_string(overflows) + " enqueued frame(s) emitted more pairs than their buffer held; "
                    "the buffers are grown, draw them again");
    if (timeouts != 0) return fail(r, LRT_TIMEOUT, "a bounded device wait gave up in an enqueued frame");
    return LRT_OK;
}

}  // namespace

extern "C" {

int lrt_rast_render(lrt_rast* r, const lrt_projection* pr, const lrt_splat_instance* instances, uint32_t n,
                    const lrt_render_settings* s, lrt_targets* targets, lrt_frame_stats* stats, void* streamPtr) {
    const auto frameStart = std::chrono::steady_clock::now();
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (pr == nullptr || s == nullptr || targets == nullptr || (n > 0 && instances == nullptr))
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    std::vector<CloudDesc> clouds;
    if (const int code = collect_clouds(r, instances, n, clouds); code != LRT_OK) return code;
    const int code = render_frame(r, pr, clouds, s, targets, stats, streamPtr, false, frameStart);
    if (code == LRT_OK) {   // a frame that waited sizes the buffers for its shape
        r->plainSized = true;
        r->plainSlots = total_slots(clouds);
        r->plainWidth = s->width;
        r->plainHeight = s->height;
        r->plainSeenPairs = r->debug.pairs_count;
    }
    return code;
}

int lrt_rast_render_composite(lrt_rast* r, const lrt_projection* pr, const lrt_splat_instance* instances, uint32_t n,
                              const lrt_point_instance* points, uint32_t pointCount, const lrt_targets* under,
                              const lrt_render_settings* s, lrt_targets* targets, lrt_frame_stats* stats,
                              void* streamPtr) {
    const auto frameStart = std::chrono::steady_clock::now();
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (pr == nullptr || s == nullptr || targets == nullptr || (n > 0 && instances == nullptr) ||
        (pointCount > 0 && points == nullptr))
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    // TileRasterizer.cpp:211-213
    if (under != nullptr && (under->width != s->width || under->height != s->height || under->colour == nullptr ||
                             under->depth == nullptr))
        return fail(r, LRT_INVALID_ARGUMENT, "the under-layer is not the frame's size");
    std::vector<CloudDesc> clouds;
    if (const int code = collect_clouds(r, instances, n, clouds); code != LRT_OK) return code;
    for (uint32_t k = 0; k < pointCount; ++k) {
        const lrt_gpu_points* g = points[k].points;
        if (g == nullptr || g->count == 0) continue;
        if (g->positions == nullptr || (reinterpret_cast<uintptr_t>(g->positions) & 15u) != 0 ||
            (points[k].style.constant_colour == 0 &&
             (g->colours == nullptr || (reinterpret_cast<uintptr_t>(g->colours) & 7u) != 0)))
            return fail(r, LRT_INVALID_ARGUMENT, "points need 16-byte aligned positions and 8-byte aligned colours");
        CloudDesc d;
        d.point = &points[k];
        d.objectToWorld = points[k].object_to_world;
        d.count = g->count;
        clouds.push_back(d);
    }
    const bool composite = under != nullptr || pointCount > 0;
    return render_frame(r, pr, clouds, s, targets, stats, streamPtr, false, frameStart, false, under, composite);
}

}  // extern "C"

namespace {

// The percentiles the reference takes from a 256-bin histogram
// (ReferenceRenderer.cpp:276-296): the bin where the running count reaches
// pixels - pixels / 100, and the highest non-empty bin.
void histogram_stats(const uint32_t* h, uint64_t& pixels, uint32_t& p99, uint32_t& maxBin, uint64_t* over2) {
    pixels = 0;
    maxBin = 0;
    uint64_t o2 = 0;
    for (uint32_t k = 0; k < 256; ++k) {
        pixels += h[k];
        if (h[k] > 0) maxBin = k;
        if (k > 2) o2 += h[k];
    }
    if (over2 != nullptr) *over2 = o2;
    const uint64_t at = pixels - pixels / 100;
    uint64_t running = 0;
    p99 = 0;
    for (uint32_t k = 0; k < 256; ++k) {
        running += h[k];
        if (running >= at) {
            p99 = k;
            break;
        }
    }
}

}  // namespace

extern "C" {

int lrt_rast_l1_loss(lrt_rast* r, const void* colour, const void* target, uint32_t pixels, void* loss,
                     void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (loss == nullptr || (pixels > 0 && (colour == nullptr || target == nullptr)))
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    LRT_CUDA(r, ensure(r->lossScratch, lrt::l1_scratch_bytes()), "loss scratch");
    LRT_CUDA(r,
             lrt::launch_l1_loss(static_cast<const float4*>(colour), static_cast<const float*>(target), pixels,
                                 static_cast<float*>(r->lossScratch.ptr), static_cast<float*>(loss), stream),
             "loss");
    return LRT_OK;
}

int lrt_l1_loss_grad(const void* colour, const void* target, uint32_t pixels, const void* gradLoss, void* gradColour,
                     void* streamPtr) {
    if (pixels > 0 && (colour == nullptr || target == nullptr || gradColour == nullptr)) return LRT_INVALID_ARGUMENT;
    const cudaError_t e = lrt::launch_l1_grad(static_cast<const float4*>(colour), static_cast<const float*>(target),
                                              pixels, static_cast<const float*>(gradLoss),
                                              static_cast<float4*>(gradColour), static_cast<cudaStream_t>(streamPtr));
    return e == cudaSuccess ? LRT_OK : LRT_DEVICE_FAILURE;
}

int lrt_rast_compare_images(lrt_rast* r, const void* a, const void* b, uint32_t width, uint32_t height,
                            lrt_image_difference* out, uint32_t* histogram, void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (out == nullptr || (uint64_t{width} * height > 0 && (a == nullptr || b == nullptr)))
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    if (uint64_t{width} * height > 0xFFFFFFFFull) return fail(r, LRT_UNSUPPORTED, "more than 2^32 pixels");
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    LRT_CUDA(r, ensure(r->metricScratch, 256 * 4 + 16), "metric scratch");
    uint32_t* bins = static_cast<uint32_t*>(r->metricScratch.ptr);
    LRT_CUDA(r, cudaMemsetAsync(bins, 0, 256 * 4, stream), "histogram");
    LRT_CUDA(r,
             lrt::launch_compare_images(static_cast<const float4*>(a), static_cast<const float4*>(b), width * height,
                                        bins, stream),
             "compare");
    LRT_CUDA(r, ensure_host(r, 256 * 4 + 16), "metric readback");
    LRT_CUDA(r, cudaMemcpyAsync(r->metricHost, bins, 256 * 4, cudaMemcpyDeviceToHost, stream), "readback");
    LRT_CUDA(r, cudaStreamSynchronize(stream), "compare");
    const uint32_t* h = static_cast<const uint32_t*>(r->metricHost);
    *out = lrt_image_difference{};
    histogram_stats(h, out->pixels, out->p99, out->max, &out->over2);
    if (histogram != nullptr) std::memcpy(histogram, h, 256 * 4);
    return LRT_OK;
}

int lrt_rast_compare_hdr(lrt_rast* r, const void* a, const void* b, uint32_t width, uint32_t height,
                         lrt_hdr_difference* out, void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (out == nullptr || (uint64_t{width} * height > 0 && (a == nullptr || b == nullptr)))
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    if (uint64_t{width} * height > 0xFFFFFFFFull) return fail(r, LRT_UNSUPPORTED, "more than 2^32 pixels");
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    const size_t bytes = 256 * 4 + 16 + size_t{height} * 4;
    LRT_CUDA(r, ensure(r->metricScratch, bytes), "metric scratch");
    uint32_t* bins = static_cast<uint32_t*>(r->metricScratch.ptr);
    float* total = reinterpret_cast<float*>(bins + 256);
    float* rows = reinterpret_cast<float*>(bins + 260);
    LRT_CUDA(r, cudaMemsetAsync(bins, 0, 256 * 4 + 16, stream), "histogram");
    LRT_CUDA(r,
             lrt::launch_compare_hdr(static_cast<const float4*>(a), static_cast<const float4*>(b), width, height, bins,
                                     rows, total, stream),
             "compare");
    LRT_CUDA(r, ensure_host(r, 256 * 4 + 16), "metric readback");
    LRT_CUDA(r, cudaMemcpyAsync(r->metricHost, bins, 256 * 4 + 4, cudaMemcpyDeviceToHost, stream), "readback");
    LRT_CUDA(r, cudaStreamSynchronize(stream), "compare");
    const uint32_t* h = static_cast<const uint32_t*>(r->metricHost);
    float error = 0.0f;
    std::memcpy(&error, h + 256, 4);
    uint32_t p99 = 0, maxBin = 0;
    *out = lrt_hdr_difference{};
    histogram_stats(h, out->pixels, p99, maxBin, nullptr);
    // Bin k > 0 holds relative differences in [2^((k-1)/8 - 16), 2^(k/8 - 16)) (ReferenceRenderer.cpp:339-360).
    const auto upper = [](uint32_t bin) { return bin == 0 ? 0.0 : std::pow(2.0, bin / 8.0 - 16.0); };
    out->max_relative = out->pixels > 0 ? upper(maxBin) : 0.0;
    out->p99_relative = out->pixels > 0 ? upper(p99) : 0.0;
    out->rel_mse = out->pixels > 0 ? static_cast<double>(error) / static_cast<double>(out->pixels) : 0.0;
    return LRT_OK;
}

int lrt_rast_count_different(lrt_rast* r, const void* a, const void* b, uint32_t count, uint64_t* out,
                             void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (out == nullptr || (count > 0 && (a == nullptr || b == nullptr)))
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    *out = 0;
    if (count == 0) return LRT_OK;
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    LRT_CUDA(r, ensure(r->metricScratch, 256 * 4 + 16), "metric scratch");
    uint64_t* total = static_cast<uint64_t*>(r->metricScratch.ptr);
    LRT_CUDA(r, cudaMemsetAsync(total, 0, 8, stream), "count");
    LRT_CUDA(r,
             lrt::launch_count_different(static_cast<const uint32_t*>(a), static_cast<const uint32_t*>(b), count,
                                         total, stream),
             "count");
    LRT_CUDA(r, ensure_host(r, 256 * 4 + 16), "metric readback");
    LRT_CUDA(r, cudaMemcpyAsync(r->metricHost, total, 8, cudaMemcpyDeviceToHost, stream), "readback");
    LRT_CUDA(r, cudaStreamSynchronize(stream), "count");
    std::memcpy(out, r->metricHost, 8);
    return LRT_OK;
}

int lrt_rast_decode_splats(lrt_rast* r, const void* raw, uint32_t count, const lrt_splat_encoding* e,
                           uint32_t keep, void* positions, void* shape, void* sh, uint32_t* kept, void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (e == nullptr || kept == nullptr ||
        (count > 0 && (raw == nullptr || positions == nullptr || shape == nullptr || sh == nullptr)))
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    *kept = 0;
    if (keep > e->rest_per_colour || !(keep == 0 || keep == 3 || keep == 8 || keep == 15))
        return fail(r, LRT_INVALID_ARGUMENT, "keep_per_colour must be 0, 3, 8 or 15 and at most the file's");
    const uint32_t fields[] = {e->x, e->y, e->z, e->opacity, e->scale0, e->scale1, e->scale2, e->rot_w, e->rot_x,
                               e->rot_y, e->rot_z, e->dc0, e->dc1, e->dc2};
    for (uint32_t f : fields)
        if (f >= e->floats_per_record) return fail(r, LRT_INVALID_ARGUMENT, "a field lies past the record");
    const uint64_t restEnd = uint64_t{e->rest_base} + 3ull * e->rest_per_colour;
    if (e->rest_per_colour > 0 && restEnd > e->floats_per_record)
        return fail(r, LRT_INVALID_ARGUMENT, "the rest coefficients lie past the record");
    if ((reinterpret_cast<uintptr_t>(positions) & 15u) != 0 || (reinterpret_cast<uintptr_t>(shape) & 15u) != 0)
        return fail(r, LRT_INVALID_ARGUMENT, "positions and shape must be 16-byte aligned");
    if (count == 0) return LRT_OK;
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    const size_t bytes = lrt::decode_status_bytes(count);
    LRT_CUDA(r, ensure(r->scanScratch, bytes), "decode scratch");
    uint32_t* err = static_cast<uint32_t*>(r->counters.ptr) + 3;
    LRT_CUDA(r, cudaMemsetAsync(r->scanScratch.ptr, 0, bytes, stream), "decode scratch");
    LRT_CUDA(r, cudaMemsetAsync(err, 0, 4, stream), "status");
    const uint32_t shWords = std::max<uint32_t>((keep * 3 + 1) / 2, 1);
    LRT_CUDA(r,
             lrt::launch_decode_splats(static_cast<const float*>(raw), count, *e, keep, shWords,
                                       static_cast<float4*>(positions), static_cast<uint4*>(shape),
                                       static_cast<uint32_t*>(sh), r->scanScratch.ptr, err, stream),
             "decode");
    const uint32_t* total = reinterpret_cast<const uint32_t*>(static_cast<char*>(r->scanScratch.ptr) + bytes - 16) + 1;
    LRT_CUDA(r, cudaMemcpyAsync(r->hostCounters + 8, total, 4, cudaMemcpyDeviceToHost, stream), "readback");
    LRT_CUDA(r, cudaMemcpyAsync(r->hostCounters + 9, err, 4, cudaMemcpyDeviceToHost, stream), "readback");
    LRT_CUDA(r, cudaStreamSynchronize(stream), "decode");
    if (r->hostCounters[9] & lrt::kErrTimeout) return fail(r, LRT_TIMEOUT, "decode look-back gave up");
    *kept = r->hostCounters[8];
    return LRT_OK;
}

int lrt_rast_decode_points(lrt_rast* r, const void* raw, uint32_t count, uint32_t colourKind, float detail,
                           void* positions, void* colours, uint32_t* kept, void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (kept == nullptr || (count > 0 && (raw == nullptr || positions == nullptr || colours == nullptr)))
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    *kept = 0;
    if (colourKind > 2) return fail(r, LRT_INVALID_ARGUMENT, "colour_kind must be 0, 1 or 2");
    if ((reinterpret_cast<uintptr_t>(positions) & 15u) != 0 || (reinterpret_cast<uintptr_t>(colours) & 7u) != 0)
        return fail(r, LRT_INVALID_ARGUMENT, "positions must be 16-byte and colours 8-byte aligned");
    if (count == 0) return LRT_OK;
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    const size_t bytes = lrt::decode_status_bytes(count);
    LRT_CUDA(r, ensure(r->scanScratch, bytes), "decode scratch");
    uint32_t* err = static_cast<uint32_t*>(r->counters.ptr) + 3;
    LRT_CUDA(r, cudaMemsetAsync(r->scanScratch.ptr, 0, bytes, stream), "decode scratch");
    LRT_CUDA(r, cudaMemsetAsync(err, 0, 4, stream), "status");
    LRT_CUDA(r,
             lrt::launch_decode_points(static_cast<const float*>(raw), count, colourKind, detail,
                                       static_cast<float4*>(positions), static_cast<uint32_t*>(colours),
                                       r->scanScratch.ptr, err, stream),
             "decode");
    const uint32_t* total = reinterpret_cast<const uint32_t*>(static_cast<char*>(r->scanScratch.ptr) + bytes - 16) + 1;
    LRT_CUDA(r, cudaMemcpyAsync(r->hostCounters + 8, total, 4, cudaMemcpyDeviceToHost, stream), "readback");
    LRT_CUDA(r, cudaMemcpyAsync(r->hostCounters + 9, err, 4, cudaMemcpyDeviceToHost, stream), "readback");
    LRT_CUDA(r, cudaStreamSynchronize(stream), "decode");
    if (r->hostCounters[9] & lrt::kErrTimeout) return fail(r, LRT_TIMEOUT, "decode look-back gave up");
    *kept = r->hostCounters[8];
    return LRT_OK;
}

int lrt_rast_render_async(lrt_rast* r, const lrt_projection* pr, const lrt_splat_instance* instances, uint32_t n,
                          const lrt_render_settings* s, lrt_targets* targets, void* streamPtr) {
    const auto frameStart = std::chrono::steady_clock::now();
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (pr == nullptr || s == nullptr || targets == nullptr || (n > 0 && instances == nullptr))
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    std::vector<CloudDesc> clouds;
    if (const int code = collect_clouds(r, instances, n, clouds); code != LRT_OK) return code;
    DeviceScope scope(r->device);
    while (r->ringTail < r->ringHead && read_oldest(r, false)) {
    }
    if (r->ringHead - r->ringTail == lrt_rast::kRing && !read_oldest(r, true))
        return fail(r, LRT_DEVICE_FAILURE, "waiting for an enqueued frame failed");
    // Enqueued only when a frame of this shape has run with a wait and the
    // last counts read leave a quarter of the pair buffer free; otherwise the
    // frame waits (and draws again with grown buffers if it has to). A frame
    // of a known shape whose last counts leave less than that grows the
    // buffer first, so that the frames after it are enqueued again.
    const uint32_t slots = total_slots(clouds);
    const uint64_t wanted = uint64_t{r->plainSeenPairs} + r->plainSeenPairs / 4;
    const bool sameShape = r->plainSized && r->plainSlots == slots && r->plainWidth == s->width &&
                           r->plainHeight == s->height;
    const bool deferred = sameShape && !s->time_stages && wanted <= r->pairCap;
    if (sameShape && !s->time_stages && wanted > r->pairCap)
        r->pairCap = grow(r->pairCap, static_cast<uint32_t>(std::min<uint64_t>(wanted, 0xFFFFFFFFull)));
    if (!deferred) {
        lrt_frame_stats stats{};
        const int code = render_frame(r, pr, clouds, s, targets, &stats, streamPtr, false, frameStart);
        if (code == LRT_OK) {
            r->plainSized = true;
            r->plainSlots = slots;
            r->plainWidth = s->width;
            r->plainHeight = s->height;
            r->plainSeenPairs = stats.pairs;
            r->asyncSplats = stats.splats;
            r->asyncVisible = stats.visible;
            r->asyncPairs = stats.pairs;
        }
        return code;
    }
    r->asyncSplats = slots;
    return render_frame(r, pr, clouds, s, targets, nullptr, streamPtr, false, frameStart, true);
}

int lrt_rast_settle(lrt_rast* r, lrt_frame_stats* stats) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    const int code = settle_async(r);
    if (stats != nullptr) {
        std::memset(stats, 0, sizeof(*stats));
        stats->splats = r->asyncSplats;
        stats->visible = r->asyncVisible;
        stats->pairs = r->asyncPairs;
    }
    return code;
}

int lrt_rast_train_forward(lrt_rast* r, const lrt_projection* pr, const lrt_train_params* params,
                           const lrt_render_settings* s, lrt_targets* targets, lrt_frame_stats* stats,
                           void* streamPtr) {
    const auto frameStart = std::chrono::steady_clock::now();
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    r->trainReady = false;
    if (pr == nullptr || params == nullptr || s == nullptr || targets == nullptr)
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    std::vector<CloudDesc> clouds;
    if (params->count > 0) {
        if (params->means == nullptr || params->log_scales == nullptr || params->quats == nullptr ||
            params->opacity_logits == nullptr || params->sh == nullptr)
            return fail(r, LRT_INVALID_ARGUMENT, "a null parameter buffer");
        if ((reinterpret_cast<uintptr_t>(params->quats) & 15u) != 0 || (reinterpret_cast<uintptr_t>(params->sh) & 15u) != 0)
            return fail(r, LRT_INVALID_ARGUMENT, "quats and sh must be 16-byte aligned");
        CloudDesc d;
        d.train = params;
        d.objectToWorld = kIdentity;
        d.count = params->count;
        clouds.push_back(d);
    }
    r->trainParams = *params;
    // A training frame waits (and redraws if its pairs overflowed) when it is
    // the first of its shape, when stage times are asked for, or when the last
    // frame whose counts were read left less than a quarter of the pair buffer
    // free. Otherwise it is only enqueued; the backward reads its counts, and
    // an overflow is reported there (and by the debug view) as OVERFLOW, with
    // the buffers grown for the next try.
    const bool sameShape = r->trainSized && r->trainSlots == params->count && r->trainWidth == s->width &&
                           r->trainHeight == s->height;
    const uint64_t wanted = uint64_t{r->trainSeenPairs} + r->trainSeenPairs / 4;
    const bool deferred = sameShape && !s->time_stages && wanted <= r->pairCap;
    if (sameShape && wanted > r->pairCap) r->pairCap = grow(r->pairCap, static_cast<uint32_t>(std::min<uint64_t>(wanted, 0xFFFFFFFFull)));
    const int code = render_frame(r, pr, clouds, s, targets, stats, streamPtr, true, frameStart, deferred);
    if (code == LRT_OK && !deferred) {
        r->trainSized = true;
        r->trainSlots = params->count;
        r->trainWidth = s->width;
        r->trainHeight = s->height;
        r->trainSeenPairs = r->trainPairs;
    }
    return code;
}

// Reads the counts of an enqueued training frame once its stream has drained:
// LRT_OVERFLOW (buffers grown, the frame must be drawn again) or LRT_TIMEOUT.
static int settle_pending_frame(lrt_rast* r) {
    r->trainPending = false;
    const uint32_t pairs = r->hostCounters[1], status = r->hostCounters[2];
    r->trainPairs = std::min(pairs, r->pairCap);
    r->trainSeenPairs = pairs;
    r->debug.pairs_count = std::min(pairs, r->pairCap);
    r->debug.visible = r->hostCounters[0];
    if (pairs > r->pairCap) {
        r->pairCap = grow(r->pairCap, pairs);
        r->trainReady = false;
        return fail(r, LRT_OVERFLOW, "the training forward emitted more pairs than its buffer held; "
                                     "the buffers are grown, run the step again");
    }
    if (status & lrt::kErrTimeout) {
        r->trainReady = false;
        return fail(r, LRT_TIMEOUT, "a bounded device wait gave up");
    }
    return LRT_OK;
}

int lrt_rast_train_backward(lrt_rast* r, const void* gradColour, lrt_train_grads* grads, void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (gradColour == nullptr || grads == nullptr) return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    if (!r->trainReady) return fail(r, LRT_INVALID_ARGUMENT, "no training forward to differentiate on this handle");
    const lrt_train_params& p = r->trainParams;
    if (p.count > 0 && (grads->means == nullptr || grads->log_scales == nullptr || grads->quats == nullptr ||
                        grads->opacity_logits == nullptr || grads->sh == nullptr))
        return fail(r, LRT_INVALID_ARGUMENT, "a null gradient buffer");
    if ((reinterpret_cast<uintptr_t>(grads->sh) & 15u) != 0)
        return fail(r, LRT_INVALID_ARGUMENT, "the SH gradient must be 16-byte aligned");
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    // A forward that ran without waiting has not reported its pair count yet:
    // the backward is enqueued over the pair buffer's capacity (every read
    // stays inside the buffers), and the forward's counts are read once the
    // backward is queued behind it, so the device never waits for the host
    // here. If that frame overflowed, the call returns OVERFLOW and the
    // gradients it wrote are not to be used.
    const bool pending = r->trainPending;
    const uint32_t pairBound = pending ? r->pairCap : r->trainPairs;
    // Every pair's partials are written by the blend backward (zeros for those
    // it does not walk), so the buffer is not cleared.
    const size_t partialBytes = std::max<size_t>(size_t{pairBound} * 12 * sizeof(float), 16);
    LRT_CUDA(r, ensure(r->partials, partialBytes), "partials");
    LRT_CUDA(r, cudaEventRecord(r->ev[7], stream), "event");
    // The backward takes the tiles busiest first by its own work: the pairs
    // up to each tile's last contributor.
    const BlendParams& tb = r->trainBlend;
    const uint32_t bTiles = tb.tilesX * tb.tilesY;
    const lrt::ChainScope chain(uint64_t{tb.width} * tb.height >= lrt::kChainMinPixels);
    uint32_t* bOrder = static_cast<uint32_t*>(r->tileOrder.ptr);
    uint32_t* bScratch = bOrder + bTiles;
    uint32_t* bWork = bScratch + lrt::tile_order_scratch_bytes(bTiles) / 4;
    LRT_CUDA(r,
             lrt::launch_tile_backward_order(static_cast<uint2*>(r->ranges.ptr), static_cast<uint32_t*>(r->pixLast.ptr),
                                             tb.width, tb.height, tb.tilesX, bTiles, bOrder, bScratch, bWork, stream),
             "backward tile order");
    LRT_CUDA(r,
             lrt::launch_blend_backward(r->trainBlend, static_cast<uint2*>(r->ranges.ptr), r->trainSorted,
                                        r->trainSortedValues, r->trainEmitSlot, static_cast<ProjRecord*>(r->proj.ptr),
                                        static_cast<float4*>(r->pixState.ptr), static_cast<uint32_t*>(r->pixLast.ptr),
                                        static_cast<const float4*>(gradColour), static_cast<float*>(r->partials.ptr),
                                        stream, bOrder),
             "blend backward");
    LRT_CUDA(r, cudaEventRecord(r->ev[8], stream), "event");
    LRT_CUDA(r,
             lrt::launch_splat_backward(r->trainFrame, static_cast<const float*>(p.means),
                                        static_cast<const float*>(p.log_scales), static_cast<const float*>(p.quats),
                                        static_cast<const float*>(p.opacity_logits),
                                        static_cast<const uint16_t*>(p.sh), static_cast<uint32_t*>(r->touched.ptr),
                                        static_cast<uint32_t*>(r->pairOffsets.ptr),
                                        static_cast<float*>(r->partials.ptr), pairBound,
                                        static_cast<float*>(grads->means),
                                        static_cast<float*>(grads->log_scales), static_cast<float*>(grads->quats),
                                        static_cast<float*>(grads->opacity_logits), static_cast<float*>(grads->sh),
                                        stream),
             "projection backward");
    LRT_CUDA(r, cudaEventRecord(r->ev[9], stream), "event");
    // The gradients are ready in stream order. Later calls on the handle (any
    // stream) wait for this event before touching its buffers.
    LRT_CUDA(r, cudaEventRecord(r->frameDone, stream), "event");
    r->frameDoneSet = true;
    r->backwardTimed = true;
    if (pending) {
        LRT_CUDA(r, cudaEventSynchronize(r->ev[6]), "frame");
        const int code = settle_pending_frame(r);
        if (code != LRT_OK) return code;
    }
    return LRT_OK;
}

int lrt_rast_backward_times(const lrt_rast* r, double* blendMs, double* projectMs) {
    if (r == nullptr || blendMs == nullptr || projectMs == nullptr) return LRT_INVALID_ARGUMENT;
    *blendMs = 0.0;
    *projectMs = 0.0;
    if (!r->backwardTimed) return LRT_OK;
    DeviceScope scope(r->device);
    if (cudaEventSynchronize(r->ev[9]) != cudaSuccess) return LRT_DEVICE_FAILURE;
    *blendMs = event_ms(r->ev[7], r->ev[8]);
    *projectMs = event_ms(r->ev[8], r->ev[9]);
    return LRT_OK;
}

int lrt_rast_debug_view(lrt_rast* r, lrt_debug_view* out) {
    if (r == nullptr || out == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (r->ringTail < r->ringHead) {   // enqueued plain frames: wait for them
        const int code = settle_async(r);
        if (code != LRT_OK) return code;
    }
    if (r->trainPending) {   // an enqueued training frame: wait for its counts
        DeviceScope scope(r->device);
        LRT_CUDA(r, cudaStreamSynchronize(r->pendingStream), "frame");
        const int code = settle_pending_frame(r);
        if (code != LRT_OK) return code;
    }
    *out = r->debug;
    return LRT_OK;
}

int lrt_prefix_sum(lrt_rast* r, const void* in, void* out, void* total, uint32_t count, void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if ((count > 0 && (in == nullptr || out == nullptr)) || total == nullptr)
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    uint32_t* err = static_cast<uint32_t*>(r->counters.ptr) + 3;
    LRT_CUDA(r, ensure(r->scanScratch, lrt::scan_scratch_bytes(count)), "scan scratch");
    LRT_CUDA(r, cudaMemsetAsync(err, 0, 4, stream), "status");
    LRT_CUDA(r,
             lrt::launch_exclusive_scan(static_cast<const uint32_t*>(in), static_cast<uint32_t*>(out),
                                        static_cast<uint32_t*>(total), count, r->scanScratch.ptr, err, stream),
             "prefix sum");
    LRT_CUDA(r, cudaMemcpyAsync(r->hostCounters + 5, err, 4, cudaMemcpyDeviceToHost, stream), "status readback");
    LRT_CUDA(r, cudaStreamSynchronize(stream), "prefix sum");
    if (r->hostCounters[5] & lrt::kErrTimeout) return fail(r, LRT_TIMEOUT, "prefix sum look-back gave up");
    if (r->hostCounters[5] & lrt::kErrTooManyPairs) return fail(r, LRT_OVERFLOW, "the sum passed 2^32 - 1");
    return LRT_OK;
}

int lrt_radix_sort(lrt_rast* r, void* keys, void* values, uint32_t count, uint32_t keyBits, uint32_t keyBytes,
                   void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (keyBytes != 4 && keyBytes != 8) return fail(r, LRT_INVALID_ARGUMENT, "key_bytes must be 4 or 8");
    if (keyBits == 0 || keyBits > keyBytes * 8) return fail(r, LRT_INVALID_ARGUMENT, "key_bits out of range");
    if (count > 0 && keys == nullptr) return fail(r, LRT_INVALID_ARGUMENT, "null keys");
    if (count <= 1) return LRT_OK;
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    uint32_t* counters = static_cast<uint32_t*>(r->counters.ptr);
    uint32_t* err = counters + 3;
    LRT_CUDA(r, ensure(r->algoKeysAlt, size_t{count} * keyBytes), "sort buffers");
    if (values != nullptr) LRT_CUDA(r, ensure(r->algoValsAlt, size_t{count} * 4), "sort buffers");
    LRT_CUDA(r, ensure(r->sortScratch, lrt::sort_scratch_bytes(count, keyBits)), "sort scratch");
    // The count lives on the device so the kernels can be replayed; write it.
    r->hostCounters[6] = count;
    LRT_CUDA(r, cudaMemcpyAsync(counters + 4, r->hostCounters + 6, 4, cudaMemcpyHostToDevice, stream), "count");
    LRT_CUDA(r, cudaMemsetAsync(err, 0, 4, stream), "status");
    bool inAlt = false;
    uint32_t* vals = static_cast<uint32_t*>(values);
    uint32_t* valsAlt = values != nullptr ? static_cast<uint32_t*>(r->algoValsAlt.ptr) : nullptr;
    if (keyBytes == 8) {
        LRT_CUDA(r,
                 lrt::launch_sort_u64(static_cast<uint64_t*>(keys), static_cast<uint64_t*>(r->algoKeysAlt.ptr), vals,
                                      valsAlt, counters + 4, count, 0, keyBits, r->sortScratch.ptr, err, &inAlt,
                                      stream, &r->sortFault),
                 "radix sort");
    } else {
        LRT_CUDA(r,
                 lrt::launch_sort_u32(static_cast<uint32_t*>(keys), static_cast<uint32_t*>(r->algoKeysAlt.ptr), vals,
                                      valsAlt, counters + 4, count, 0, keyBits, r->sortScratch.ptr, err, &inAlt,
                                      stream, &r->sortFault),
                 "radix sort");
    }
    if (inAlt) {   // an odd pass count ends in the scratch buffers (RadixSort.cpp:146-155 copies back too)
        LRT_CUDA(r, cudaMemcpyAsync(keys, r->algoKeysAlt.ptr, size_t{count} * keyBytes, cudaMemcpyDeviceToDevice, stream),
                 "copy back");
        if (values != nullptr)
            LRT_CUDA(r, cudaMemcpyAsync(values, r->algoValsAlt.ptr, size_t{count} * 4, cudaMemcpyDeviceToDevice, stream),
                     "copy back");
    }
    LRT_CUDA(r, cudaMemcpyAsync(r->hostCounters + 7, err, 4, cudaMemcpyDeviceToHost, stream), "status readback");
    LRT_CUDA(r, cudaStreamSynchronize(stream), "radix sort");
    if (r->hostCounters[7] & lrt::kErrTimeout) return fail(r, LRT_TIMEOUT, "radix sort look-back gave up");
    return LRT_OK;
}

int lrt_rast_debug_sort(lrt_rast* r, uint32_t skip_first_partition, uint32_t poll_limit, uint32_t wide_look_back) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    r->sortFault.skipFirstPartition = skip_first_partition != 0 ? 1u : 0u;
    r->sortFault.pollLimit = poll_limit;
    r->sortFault.wideWords = wide_look_back != 0 ? 1u : 0u;
    return LRT_OK;
}

}  // extern "C"

// --------------------------------------------------------------- batches ----
namespace {

struct BatchShape {
    std::vector<uint32_t> order;   // views, largest first
    uint32_t slots = 0, launchesPerView = 0;
    uint64_t key = 0;
};

uint64_t mix(uint64_t h, uint64_t v) {
    h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    return h;
}

// Grows a buffer and, when it moves, invalidates the batch graph.
cudaError_t ensure_batch(lrt_rast* r, DeviceBuffer& b, size_t bytes) {
    if (b.bytes >= bytes && b.ptr != nullptr) return cudaSuccess;
    r->batch.generation += 1;
    return ensure(b, bytes);
}

// Enqueues the whole batch (all chunks) on the batch stream. Host-side
// parameters must already be in batch.hostParams; the first operation copies
// them to the device, so a captured graph replays with whatever cameras the
// pinned buffer holds at launch.
int enqueue_batch(lrt_rast* r, const std::vector<CloudDesc>& clouds, const lrt_view* views, const BatchShape& shape,
                  const lrt_render_settings* s, uint32_t perChunk, uint32_t blocksPerSM, uint32_t numSMs) {
    auto& B = r->batch;
    const uint32_t nViews = static_cast<uint32_t>(shape.order.size());
    const uint32_t nLaunch = nViews * shape.launchesPerView;
    const size_t paramsBytes = view_params_offset(nLaunch) + size_t{nViews} * sizeof(lrt::ViewParams);
    LRT_CUDA(r, cudaMemcpyAsync(B.params.ptr, B.hostParams, paramsBytes, cudaMemcpyHostToDevice, B.stream), "params");
    const FrameParams* devF = static_cast<const FrameParams*>(B.params.ptr);
    const lrt::ViewParams* devV = reinterpret_cast<const lrt::ViewParams*>(static_cast<const char*>(B.params.ptr) +
                                                                          view_params_offset(nLaunch));
    const FrameParams* hostF = static_cast<const FrameParams*>(B.hostParams);
    const lrt::ViewParams* hostV = reinterpret_cast<const lrt::ViewParams*>(static_cast<const char*>(B.hostParams) +
                                                                           view_params_offset(nLaunch));
    const uint32_t slotBits = bits_for(std::max<uint32_t>(shape.slots, 1));
    BlendParams bp{};
    bp.slotBits = slotBits;
    bp.tileShift = 24 + slotBits;
    bp.depthMode = s->depth_mode;
    bp.linearise = s->linearise ? 1u : 0u;
    bp.depthThreshold = s->depth_threshold;
    for (int a = 0; a < 4; ++a) bp.bg[a] = s->background[a];
    uint32_t chunk = 0;
    for (uint32_t v0 = 0; v0 < nViews; v0 += perChunk, ++chunk) {
        const uint32_t v1 = std::min(nViews, v0 + perChunk);
        uint32_t chunkTiles = 0;
        uint64_t partitions = 0;
        for (uint32_t v = v0; v < v1; ++v) {
            chunkTiles += hostV[v].tilesX * ((hostV[v].height + lrt::kTile - 1) / lrt::kTile);
            for (const CloudDesc& c : clouds) partitions += lrt::project_partitions(c.count);
        }
        const uint32_t keyBits = 24 + bits_for(chunkTiles);
        uint32_t* counters = static_cast<uint32_t*>(B.counters.ptr) + 4 * chunk;
        uint32_t* err = counters + 2;
        const size_t statusBytes = lrt::project_status_bytes(static_cast<uint32_t>(partitions)) +
                                   size_t{(v1 - v0) * shape.launchesPerView} * 4;
        uint64_t* status = static_cast<uint64_t*>(r->scanScratch.ptr);
        uint32_t* tickets = reinterpret_cast<uint32_t*>(static_cast<char*>(r->scanScratch.ptr) +
                                                        lrt::project_status_bytes(static_cast<uint32_t>(partitions)));
        LRT_CUDA(r, cudaMemsetAsync(counters, 0, 16, B.stream), "counters");
        LRT_CUDA(r, cudaMemsetAsync(r->scanScratch.ptr, 0, statusBytes, B.stream), "projection scratch");
        LRT_CUDA(r, cudaMemsetAsync(static_cast<uint32_t*>(B.queue.ptr) + chunk, 0, 4, B.stream), "queue");
        const uint32_t lastPartition = static_cast<uint32_t>(partitions - 1);
        uint32_t partitionBase = 0, launch = 0;
        for (uint32_t v = v0; v < v1; ++v) {
            for (uint32_t k = 0; k < shape.launchesPerView; ++k) {
                const uint32_t li = v * shape.launchesPerView + k;
                const CloudDesc& c = clouds[k];
                LRT_CUDA(r,
                         lrt::launch_project_emit(
                             hostF[li], static_cast<const float4*>(c.packed->positions),
                             static_cast<const uint4*>(c.packed->shape), static_cast<const uint32_t*>(c.packed->sh),
                             static_cast<ProjRecord*>(B.records.ptr), nullptr, nullptr, nullptr, counters, status,
                             tickets + launch, partitionBase, lastPartition, slotBits,
                             static_cast<uint64_t*>(r->pairs.ptr), r->pairCap, B.stream, devF + li,
                             static_cast<const float*>(c.packed->filter3d)),
                         "project");
                partitionBase += lrt::project_partitions(c.count);
                launch += 1;
            }
        }
        bool inAlt = false;
        LRT_CUDA(r,
                 lrt::launch_sort_u64(static_cast<uint64_t*>(r->pairs.ptr), static_cast<uint64_t*>(r->pairsAlt.ptr),
                                      nullptr, nullptr, counters + 1, r->pairCap, slotBits, keyBits,
                                      r->sortScratch.ptr, err, &inAlt, B.stream),
                 "pair sort");
        const uint64_t* sorted = inAlt ? static_cast<uint64_t*>(r->pairsAlt.ptr) : static_cast<uint64_t*>(r->pairs.ptr);
        LRT_CUDA(r,
                 lrt::launch_ranges(sorted, counters + 1, r->pairCap, 24 + slotBits, static_cast<uint2*>(B.ranges.ptr),
                                    chunkTiles, B.stream),
                 "ranges");
        LRT_CUDA(r,
                 lrt::launch_blend_batch(bp, devV + v0, v1 - v0, static_cast<uint2*>(B.ranges.ptr), sorted,
                                         static_cast<ProjRecord*>(B.records.ptr), chunkTiles,
                                         static_cast<uint32_t*>(B.queue.ptr) + chunk, err, numSMs * blocksPerSM,
                                         B.stream),
                 "blend");
        LRT_CUDA(r, cudaMemcpyAsync(B.hostCounters + 4 * chunk, counters, 16, cudaMemcpyDeviceToHost, B.stream),
                 "readback");
    }
    return LRT_OK;
}

}  // namespace

extern "C" int lrt_rast_render_batch(lrt_rast* r, const lrt_splat_instance* instances, uint32_t n,
                                     const lrt_view* views, uint32_t nViews, const lrt_render_settings* s,
                                     lrt_batch_stats* stats, void* streamPtr) {
    const auto t0 = std::chrono::steady_clock::now();
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (s == nullptr || (n > 0 && instances == nullptr) || (nViews > 0 && views == nullptr))
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    std::vector<CloudDesc> clouds;
    uint64_t total = 0;
    for (uint32_t k = 0; k < n; ++k) {
        const lrt_gpu_splats* c = instances[k].splats;
        if (c == nullptr || c->count == 0) continue;
        if (c->positions == nullptr || c->shape == nullptr || (c->rest_per_colour > 0 && c->sh == nullptr))
            return fail(r, LRT_INVALID_ARGUMENT, "a cloud without its buffers");
        CloudDesc d;
        d.packed = c;
        d.objectToWorld = instances[k].object_to_world;
        d.edit = &instances[k].edit;
        d.count = c->count;
        clouds.push_back(d);
        total += c->count;
    }
    if (total > 0xFFFFFFFFull) return fail(r, LRT_UNSUPPORTED, "more than 2^32 splats in one view");
    for (uint32_t v = 0; v < nViews; ++v) {
        if (views[v].width == 0 || views[v].height == 0) return fail(r, LRT_INVALID_ARGUMENT, "a view needs a size");
        if (views[v].width > lrt::kMaxFrameSide || views[v].height > lrt::kMaxFrameSide)
            return fail(r, LRT_UNSUPPORTED, "a view side above 2^19 pixels");
        if (views[v].colour == nullptr || views[v].depth == nullptr)
            return fail(r, LRT_INVALID_ARGUMENT, "a view without its images");
    }
    if (stats != nullptr) std::memset(stats, 0, sizeof(*stats));
    if (nViews == 0) return LRT_OK;
    DeviceScope scope(r->device);
    auto& B = r->batch;
    cudaStream_t caller = static_cast<cudaStream_t>(streamPtr);
    if (B.stream == nullptr) {
        LRT_CUDA(r, cudaStreamCreateWithFlags(&B.stream, cudaStreamNonBlocking), "batch stream");
        for (cudaEvent_t* e : {&B.in, &B.out, &B.start, &B.end}) LRT_CUDA(r, cudaEventCreate(e), "batch event");
    }
    int numSMs = 148;
    cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, r->device);

    // Shape: views largest first; everything a captured graph depends on.
    BatchShape shape;
    shape.slots = static_cast<uint32_t>(total);
    shape.launchesPerView = static_cast<uint32_t>(clouds.size());
    shape.order.resize(nViews);
    for (uint32_t v = 0; v < nViews; ++v) shape.order[v] = v;
    std::stable_sort(shape.order.begin(), shape.order.end(), [&](uint32_t a, uint32_t b) {
        return uint64_t{views[a].width} * views[a].height > uint64_t{views[b].width} * views[b].height;
    });
    uint64_t key = mix(0, nViews);
    key = mix(key, total);
    for (uint32_t v : shape.order) key = mix(mix(key, views[v].width), views[v].height);
    // Every pointer a captured launch bakes in is part of the key.
    for (const CloudDesc& c : clouds) {
        key = mix(mix(key, reinterpret_cast<uintptr_t>(c.packed->positions)), c.count);
        key = mix(mix(key, reinterpret_cast<uintptr_t>(c.packed->shape)), reinterpret_cast<uintptr_t>(c.packed->sh));
        key = mix(key, reinterpret_cast<uintptr_t>(c.packed->filter3d));
    }
    key = mix(key, (uint64_t{s->antialias} << 1) ^ (uint64_t{s->max_sh_degree} << 3) ^ (uint64_t{s->linearise} << 7) ^
                       (uint64_t{s->depth_mode} << 9));
    shape.key = key;
    if (clouds.empty() || total == 0) {
        // Nothing to draw: the background.
        for (uint32_t v = 0; v < nViews; ++v) {
            lrt_targets t{views[v].width, views[v].height, views[v].colour, views[v].depth};
            lrt_render_settings sv = *s;
            sv.width = views[v].width;
            sv.height = views[v].height;
            const int code = lrt_rast_render(r, &views[v].projection, nullptr, 0, &sv, &t, nullptr, streamPtr);
            if (code != LRT_OK) return code;
        }
        if (stats != nullptr) stats->views = nViews;
        return LRT_OK;
    }
    const uint32_t slotBits = bits_for(total);

    // Per (view, instance) projection parameters and per view blend parameters,
    // written to pinned memory in view order (largest first).
    const uint32_t nLaunch = nViews * shape.launchesPerView;
    const size_t paramsBytes = view_params_offset(nLaunch) + size_t{nViews} * sizeof(lrt::ViewParams);
    if (B.hostParamsBytes < paramsBytes) {
        if (B.hostParams != nullptr) cudaFreeHost(B.hostParams);
        B.hostParams = nullptr;
        B.hostParamsBytes = 0;
        LRT_CUDA(r, cudaMallocHost(&B.hostParams, paramsBytes), "batch parameters");
        B.hostParamsBytes = paramsBytes;
        B.generation += 1;
    }
    LRT_CUDA(r, ensure_batch(r, B.params, paramsBytes), "batch parameters");
    FrameParams* hostF = static_cast<FrameParams*>(B.hostParams);
    lrt::ViewParams* hostV = reinterpret_cast<lrt::ViewParams*>(static_cast<char*>(B.hostParams) +
                                                               view_params_offset(nLaunch));

    // The chunking the autotuner picked for this shape (tune on first sight).
    uint32_t perChunk = 0, blocksPerSM = 0;
    for (auto& t : B.tuned)
        if (t.first == key) {
            perChunk = t.second.first;
            blocksPerSM = t.second.second;
        }
    const bool tuning = perChunk == 0;

    auto fill = [&](uint32_t chunkViews) {
        // Tile numbering restarts at each chunk; records are per chunk slot.
        uint32_t tileBase = 0;
        for (uint32_t i = 0; i < nViews; ++i) {
            if (i % chunkViews == 0) tileBase = 0;
            const lrt_view& vw = views[shape.order[i]];
            lrt_render_settings sv = *s;
            sv.width = vw.width;
            sv.height = vw.height;
            const uint32_t tilesX = (vw.width + lrt::kTile - 1) / lrt::kTile;
            const uint32_t tilesY = (vw.height + lrt::kTile - 1) / lrt::kTile;
            const uint32_t recordBase = (i % chunkViews) * shape.slots;
            uint32_t base = 0;
            for (uint32_t k = 0; k < shape.launchesPerView; ++k) {
                FrameParams f = frame_params(&vw.projection, &sv, clouds[k], tilesX, tilesY, base);
                f.tileBase = tileBase;
                f.recordBase = recordBase;
                f.writeDebug = 0;
                hostF[i * shape.launchesPerView + k] = f;
                base += clouds[k].count;
            }
            lrt::ViewParams vp{};
            vp.width = vw.width;
            vp.height = vw.height;
            vp.tilesX = tilesX;
            vp.tileBase = tileBase;
            vp.recordBase = recordBase;
            vp.colour = static_cast<float4*>(vw.colour);
            vp.depth = static_cast<float*>(vw.depth);
            hostV[i] = vp;
            tileBase += tilesX * tilesY;
        }
    };

    // Buffers for a chunk size; false and an error when something failed.
    auto reserve = [&](uint32_t chunkViews) -> int {
        uint32_t maxTiles = 0, tiles = 0;
        for (uint32_t i = 0; i < nViews; ++i) {
            if (i % chunkViews == 0) tiles = 0;
            const lrt_view& vw = views[shape.order[i]];
            tiles += ((vw.width + 15) / 16) * ((vw.height + 15) / 16);
            maxTiles = std::max(maxTiles, tiles);
        }
        if (slotBits + 24 + bits_for(maxTiles) > 64)
            return fail(r, LRT_UNSUPPORTED, "splat slots and a chunk's tiles do not fit one 64-bit pair word");
        const uint64_t partitions = uint64_t{chunkViews} * [&] {
            uint64_t p = 0;
            for (const CloudDesc& c : clouds) p += lrt::project_partitions(c.count);
            return p;
        }();
        const size_t statusBytes = lrt::project_status_bytes(static_cast<uint32_t>(partitions)) +
                                   size_t{chunkViews * shape.launchesPerView} * 4;
        if (r->scanScratch.bytes < statusBytes) {
            r->batch.generation += 1;
            LRT_CUDA(r, ensure(r->scanScratch, statusBytes), "projection scratch");
        }
        LRT_CUDA(r, ensure_batch(r, B.records, size_t{chunkViews} * shape.slots * sizeof(ProjRecord)), "records");
        LRT_CUDA(r, ensure_batch(r, B.ranges, size_t{maxTiles} * 8), "ranges");
        const uint32_t chunks = (nViews + chunkViews - 1) / chunkViews;
        LRT_CUDA(r, ensure_batch(r, B.counters, size_t{chunks} * 16), "counters");
        LRT_CUDA(r, ensure_batch(r, B.queue, size_t{chunks} * 4), "queue");
        if (B.hostCounterChunks < chunks) {
            if (B.hostCounters != nullptr) cudaFreeHost(B.hostCounters);
            B.hostCounters = nullptr;
            LRT_CUDA(r, cudaMallocHost(reinterpret_cast<void**>(&B.hostCounters), size_t{chunks} * 16), "counters");
            B.hostCounterChunks = chunks;
            B.generation += 1;
        }
        if (r->pairCap == 0) {
            uint64_t pixels = 0;
            for (uint32_t i = 0; i < std::min(nViews, chunkViews); ++i)
                pixels += uint64_t{views[shape.order[i]].width} * views[shape.order[i]].height;
            r->pairCap = static_cast<uint32_t>(std::min<uint64_t>(std::max<uint64_t>(pixels, 1024), 0xFFFFFFFFull));
        }
        if (r->pairs.bytes < size_t{r->pairCap} * 8 || r->pairsAlt.bytes < size_t{r->pairCap} * 8) r->batch.generation += 1;
        LRT_CUDA(r, ensure(r->pairs, size_t{r->pairCap} * 8), "pairs");
        LRT_CUDA(r, ensure(r->pairsAlt, size_t{r->pairCap} * 8), "pairs");
        const size_t sortBytes = lrt::sort_scratch_bytes(r->pairCap, 24 + bits_for(maxTiles));
        if (r->sortScratch.bytes < sortBytes) r->batch.generation += 1;
        LRT_CUDA(r, ensure(r->sortScratch, sortBytes), "sort scratch");
        return LRT_OK;
    };

    // One eager run of the batch: returns the status, sets *overflowed and
    // the device time.
    auto eager = [&](uint32_t chunkViews, uint32_t bps, bool* overflowed, float* ms) -> int {
        for (int attempt = 0; attempt < 3; ++attempt) {
            int code = reserve(chunkViews);
            if (code != LRT_OK) return code;
            fill(chunkViews);
            LRT_CUDA(r, cudaEventRecord(B.start, B.stream), "event");
            code = enqueue_batch(r, clouds, views, shape, s, chunkViews, bps, static_cast<uint32_t>(numSMs));
            if (code != LRT_OK) return code;
            LRT_CUDA(r, cudaEventRecord(B.end, B.stream), "event");
            LRT_CUDA(r, cudaStreamSynchronize(B.stream), "batch");
            LRT_CUDA(r, cudaEventElapsedTime(ms, B.start, B.end), "event");
            const uint32_t chunks = (nViews + chunkViews - 1) / chunkViews;
            uint32_t worst = 0, statusBits = 0;
            for (uint32_t c = 0; c < chunks; ++c) {
                worst = std::max(worst, B.hostCounters[4 * c + 1]);
                statusBits |= B.hostCounters[4 * c + 2];
            }
            if (statusBits & lrt::kErrTimeout) return fail(r, LRT_TIMEOUT, "a bounded device wait gave up");
            if (statusBits & lrt::kErrTooManyPairs) return fail(r, LRT_UNSUPPORTED, "more than 2^32 pairs in a chunk");
            *overflowed = worst > r->pairCap;
            if (!*overflowed) return LRT_OK;
            r->pairCap = grow(r->pairCap, worst);
        }
        return fail(r, LRT_OVERFLOW, "pair capacity exceeded");
    };

    LRT_CUDA(r, cudaEventRecord(B.in, caller), "event");
    LRT_CUDA(r, cudaStreamWaitEvent(B.stream, B.in, 0), "event");
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(B.stream, r->frameDone, 0), "frame order");
    bool replayed = false;
    float deviceMs = 0.0f;
    if (tuning) {
        // Autotune: views per chunk x blend blocks per SM, fastest of one timed run each.
        std::vector<uint32_t> chunkSizes;
        for (uint32_t c : {nViews, 32u, 16u, 8u, 4u})
            if (c <= nViews && c >= 1 && std::find(chunkSizes.begin(), chunkSizes.end(), c) == chunkSizes.end())
                chunkSizes.push_back(c);
        float best = 3.4e38f;
        for (uint32_t c : chunkSizes) {
            for (uint32_t bps : {4u, 8u}) {
                bool over = false;
                float ms = 0.0f;
                int code = eager(c, bps, &over, &ms);   // sizes the buffers
                if (code != LRT_OK) return code;
                code = eager(c, bps, &over, &ms);
                if (code != LRT_OK) return code;
                if (ms < best) {
                    best = ms;
                    perChunk = c;
                    blocksPerSM = bps;
                }
            }
        }
        B.tuned.push_back({key, {perChunk, blocksPerSM}});
        bool over = false;
        const int code = eager(perChunk, blocksPerSM, &over, &deviceMs);   // the frame itself, with the choice
        if (code != LRT_OK) return code;
    } else {
        int code = reserve(perChunk);
        if (code != LRT_OK) return code;
        fill(perChunk);
        // The buffers the batch shares with single frames (which can move
        // them between batches) are part of what a captured graph bakes in.
        uint64_t gkey = key;
        for (const void* q : {r->pairs.ptr, r->pairsAlt.ptr, r->scanScratch.ptr, r->sortScratch.ptr})
            gkey = mix(gkey, reinterpret_cast<uintptr_t>(q));
        const bool haveGraph = B.graph != nullptr && B.graphKey == gkey && B.graphGeneration == B.generation;
        if (!haveGraph && !B.graphFailed) {
            // Capture this shape's batch into a graph.
            if (B.graph != nullptr) {
                cudaGraphExecDestroy(B.graph);
                B.graph = nullptr;
            }
            cudaGraph_t graph = nullptr;
            bool ok = cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                code = enqueue_batch(r, clouds, views, shape, s, perChunk, blocksPerSM, static_cast<uint32_t>(numSMs));
                ok = cudaStreamEndCapture(B.stream, &graph) == cudaSuccess && code == LRT_OK;
            }
            if (ok) ok = cudaGraphInstantiate(&B.graph, graph, 0) == cudaSuccess;
            if (graph != nullptr) cudaGraphDestroy(graph);
            cudaGetLastError();
            if (ok) {
                B.graphKey = gkey;
                B.graphGeneration = B.generation;
            } else {
                B.graph = nullptr;
                B.graphFailed = true;   // keep running eagerly
                r->error.clear();
            }
        }
        bool over = false;
        if (B.graph != nullptr && B.graphKey == gkey && B.graphGeneration == B.generation) {
            LRT_CUDA(r, cudaEventRecord(B.start, B.stream), "event");
            LRT_CUDA(r, cudaGraphLaunch(B.graph, B.stream), "graph launch");
            LRT_CUDA(r, cudaEventRecord(B.end, B.stream), "event");
            LRT_CUDA(r, cudaStreamSynchronize(B.stream), "batch");
            LRT_CUDA(r, cudaEventElapsedTime(&deviceMs, B.start, B.end), "event");
            const uint32_t chunks = (nViews + perChunk - 1) / perChunk;
            uint32_t worst = 0, statusBits = 0;
            for (uint32_t c = 0; c < chunks; ++c) {
                worst = std::max(worst, B.hostCounters[4 * c + 1]);
                statusBits |= B.hostCounters[4 * c + 2];
            }
            if (statusBits & lrt::kErrTimeout) return fail(r, LRT_TIMEOUT, "a bounded device wait gave up");
            over = worst > r->pairCap;
            replayed = !over;
            if (over) r->pairCap = grow(r->pairCap, worst);
        }
        if (!replayed) {
            code = eager(perChunk, blocksPerSM, &over, &deviceMs);
            if (code != LRT_OK) return code;
        }
    }
    LRT_CUDA(r, cudaEventRecord(B.out, B.stream), "event");
    LRT_CUDA(r, cudaStreamWaitEvent(caller, B.out, 0), "event");
    LRT_CUDA(r, cudaEventRecord(r->frameDone, B.stream), "event");
    r->frameDoneSet = true;
    if (stats != nullptr) {
        const uint32_t chunks = (nViews + perChunk - 1) / perChunk;
        uint64_t pairs = 0;
        for (uint32_t c = 0; c < chunks; ++c) pairs += B.hostCounters[4 * c + 1];
        stats->views = nViews;
        stats->splats = static_cast<uint32_t>(total);
        stats->pairs = static_cast<uint32_t>(std::min<uint64_t>(pairs, 0xFFFFFFFFull));
        stats->chunks = chunks;
        stats->views_per_chunk = perChunk;
        stats->blend_blocks_per_sm = blocksPerSM;
        stats->graph_replayed = replayed ? 1u : 0u;
        stats->device_ms = deviceMs;
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return LRT_OK;
}
