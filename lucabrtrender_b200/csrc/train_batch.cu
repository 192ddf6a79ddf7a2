// lrt_rast_train_batch: one training step over many views of one cloud of raw
// parameters (no reference counterpart; the reference renders one view per
// call and has no backward).
//
// Views go in chunks. Per chunk:
//   one projection launch per view (the training source, records at the
//   view's base, pair offsets and touched counts per view) into one pair
//   buffer whose tile ids number the chunk's tiles view after view -> one
//   sort of (tile | depth | slot) words carrying each pair's emit index as a
//   value -> ranges -> one persistent training blend over (view, tile) items
//   -> per view the L1 loss and its gradient -> one backward-blend launch
//   over the chunk's (view, tile) items, writing per-pair partials at their
//   emit indices -> one per-splat backward over the chunk's views: each
//   splat's gradients summed view after view (from zero in the batch's first
//   chunk, from the buffers' values in later ones) and written once.
// Each view's pixels, and each view's gradient contribution, are the same
// bits as a single-view training step of that view: within a tile the pairs
// keep the single view's order, and a splat's pairs are contiguous at their
// emit indices as in a single view.
#include "rast_handle.h"

#include <chrono>
#include <cstring>

namespace {

constexpr uint32_t kTrainChunkViews = 16;   // views per chunk (bounds the pairs and partials held at once)
constexpr uint32_t kTrainBlendBlocksPerSM = 4;

struct ChunkView {
    FrameParams f;
    lrt::ViewParams v;
    size_t pixBase;   // the view's first pixel in the chunk's pixel buffers
    uint32_t pixels;
};

}  // namespace

extern "C" int lrt_rast_train_batch(lrt_rast* r, const lrt_train_params* params, const lrt_train_view* views,
                                    uint32_t nViews, const lrt_render_settings* s, lrt_train_grads* grads,
                                    lrt_batch_stats* stats, void* streamPtr) {
    const auto t0 = std::chrono::steady_clock::now();
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (params == nullptr || s == nullptr || grads == nullptr || (nViews > 0 && views == nullptr))
        return fail(r, LRT_INVALID_ARGUMENT, "null argument");
    const uint32_t n = params->count;
    if (n == 0) return fail(r, LRT_INVALID_ARGUMENT, "a training batch needs splats");
    if (params->means == nullptr || params->log_scales == nullptr || params->quats == nullptr ||
        params->opacity_logits == nullptr || params->sh == nullptr)
        return fail(r, LRT_INVALID_ARGUMENT, "a null parameter buffer");
    if ((reinterpret_cast<uintptr_t>(params->quats) & 15u) != 0 || (reinterpret_cast<uintptr_t>(params->sh) & 15u) != 0)
        return fail(r, LRT_INVALID_ARGUMENT, "quats and sh must be 16-byte aligned");
    if (grads->means == nullptr || grads->log_scales == nullptr || grads->quats == nullptr ||
        grads->opacity_logits == nullptr || grads->sh == nullptr)
        return fail(r, LRT_INVALID_ARGUMENT, "a null gradient buffer");
    if ((reinterpret_cast<uintptr_t>(grads->sh) & 15u) != 0)
        return fail(r, LRT_INVALID_ARGUMENT, "the SH gradient must be 16-byte aligned");
    for (uint32_t v = 0; v < nViews; ++v) {
        if (views[v].width == 0 || views[v].height == 0) return fail(r, LRT_INVALID_ARGUMENT, "a view needs a size");
        if (views[v].colour == nullptr || views[v].depth == nullptr || views[v].target == nullptr)
            return fail(r, LRT_INVALID_ARGUMENT, "a view without its images or target");
    }
    if (stats != nullptr) std::memset(stats, 0, sizeof(*stats));
    if (nViews == 0) return LRT_OK;
    const uint64_t slotsPerChunk = uint64_t{std::min(nViews, kTrainChunkViews)} * n;
    if (slotsPerChunk > 0xFFFFFFFFull) return fail(r, LRT_UNSUPPORTED, "a chunk's records pass 2^32");

    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    // This step reuses the single-view training buffers: a training frame
    // still waiting for its backward is dropped.
    r->trainReady = false;
    r->trainPending = false;
    int numSMs = 148;
    cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, r->device);

    CloudDesc cloud;
    cloud.train = params;
    cloud.objectToWorld = kIdentity;
    cloud.count = n;
    const uint32_t slotBits = bits_for(n);
    const uint32_t perChunk = std::min(nViews, kTrainChunkViews);

    // Buffers for the largest chunk.
    size_t maxPixels = 0;
    uint32_t maxTiles = 0;
    for (uint32_t c0 = 0; c0 < nViews; c0 += perChunk) {
        size_t pixels = 0;
        uint32_t tiles = 0;
        for (uint32_t v = c0; v < std::min(nViews, c0 + perChunk); ++v) {
            pixels += size_t{views[v].width} * views[v].height;
            tiles += ((views[v].width + lrt::kTile - 1) / lrt::kTile) * ((views[v].height + lrt::kTile - 1) / lrt::kTile);
        }
        maxPixels = std::max(maxPixels, pixels);
        maxTiles = std::max(maxTiles, tiles);
    }
    if (slotBits + 24 + bits_for(maxTiles) > 64)
        return fail(r, LRT_UNSUPPORTED, "splat slots and a chunk's tiles do not fit one 64-bit pair word");
    const uint64_t partitions = uint64_t{perChunk} * lrt::project_partitions(n);
    const size_t statusBytes = lrt::project_status_bytes(static_cast<uint32_t>(partitions)) + size_t{perChunk} * 4;
    LRT_CUDA(r, ensure(r->proj, slotsPerChunk * sizeof(ProjRecord)), "splat records");
    LRT_CUDA(r, ensure(r->touched, slotsPerChunk * 4), "touched counts");
    LRT_CUDA(r, ensure(r->trainOffsets, slotsPerChunk * 4), "pair offsets");
    LRT_CUDA(r, ensure(r->pixState, maxPixels * 16), "pixel state");
    LRT_CUDA(r, ensure(r->pixLast, maxPixels * 4), "pixel state");
    LRT_CUDA(r, ensure(r->trainBatchGrad, maxPixels * 16), "colour gradients");
    LRT_CUDA(r, ensure(r->trainBatchViews, size_t{perChunk} * sizeof(lrt::ViewParams) + 16), "view parameters");
    LRT_CUDA(r, ensure(r->trainBatchLoss, size_t{perChunk} * 4 + 16), "losses");
    LRT_CUDA(r, ensure(r->trainBatchFrames, size_t{perChunk} * sizeof(FrameParams)), "frame parameters");
    LRT_CUDA(r, ensure(r->lossScratch, lrt::l1_scratch_bytes()), "loss scratch");
    LRT_CUDA(r, ensure(r->scanScratch, std::max<size_t>(statusBytes, 16)), "projection scratch");
    LRT_CUDA(r, ensure(r->ranges, size_t{maxTiles} * 8), "tile ranges");
    if (r->trainBatchPairCap == 0)
        r->trainBatchPairCap = std::max<uint32_t>(1024, static_cast<uint32_t>(std::min<uint64_t>(slotsPerChunk * 4, 0xFFFFFFFFull)));

    uint32_t* counters = static_cast<uint32_t*>(r->counters.ptr);
    uint32_t* err = counters + 2;
    uint64_t* status = static_cast<uint64_t*>(r->scanScratch.ptr);
    uint32_t* tickets = reinterpret_cast<uint32_t*>(static_cast<char*>(r->scanScratch.ptr) +
                                                    lrt::project_status_bytes(static_cast<uint32_t>(partitions)));
    lrt::ViewParams* devViews = static_cast<lrt::ViewParams*>(r->trainBatchViews.ptr);
    uint32_t* queue = reinterpret_cast<uint32_t*>(static_cast<char*>(r->trainBatchViews.ptr) +
                                                  size_t{perChunk} * sizeof(lrt::ViewParams));
    BlendParams bp{};
    bp.slotBits = slotBits;
    bp.tileShift = 24 + slotBits;
    bp.depthMode = s->depth_mode;
    bp.linearise = s->linearise ? 1u : 0u;
    bp.depthThreshold = s->depth_threshold;
    for (int a = 0; a < 4; ++a) bp.bg[a] = s->background[a];
    const float* means = static_cast<const float*>(params->means);
    const float* logScales = static_cast<const float*>(params->log_scales);
    const float* quats = static_cast<const float*>(params->quats);
    const float* logits = static_cast<const float*>(params->opacity_logits);
    const uint16_t* sh = static_cast<const uint16_t*>(params->sh);
    uint64_t totalPairs = 0;
    uint32_t chunks = 0;

    LRT_CUDA(r, cudaEventRecord(r->ev[6], stream), "event");
    std::vector<ChunkView> cv;
    for (uint32_t c0 = 0; c0 < nViews; c0 += perChunk, ++chunks) {
        const uint32_t c1 = std::min(nViews, c0 + perChunk);
        const uint32_t count = c1 - c0;
        cv.assign(count, ChunkView{});
        uint32_t tileBase = 0;
        size_t pixBase = 0;
        for (uint32_t k = 0; k < count; ++k) {
            const lrt_train_view& vw = views[c0 + k];
            lrt_render_settings sv = *s;
            sv.width = vw.width;
            sv.height = vw.height;
            const uint32_t tilesX = (vw.width + lrt::kTile - 1) / lrt::kTile;
            const uint32_t tilesY = (vw.height + lrt::kTile - 1) / lrt::kTile;
            ChunkView& c = cv[k];
            c.f = frame_params(&vw.projection, &sv, cloud, tilesX, tilesY, 0);
            c.f.tileBase = tileBase;
            c.f.recordBase = k * n;
            c.f.writeDebug = 0;
            c.pixBase = pixBase;
            c.pixels = vw.width * vw.height;
            c.v.width = vw.width;
            c.v.height = vw.height;
            c.v.tilesX = tilesX;
            c.v.tileBase = tileBase;
            c.v.recordBase = k * n;
            c.v.colour = static_cast<float4*>(vw.colour);
            c.v.depth = static_cast<float*>(vw.depth);
            c.v.pixState = static_cast<float4*>(r->pixState.ptr) + pixBase;
            c.v.pixLast = static_cast<uint32_t*>(r->pixLast.ptr) + pixBase;
            c.v.gradColour = static_cast<const float4*>(r->trainBatchGrad.ptr) + pixBase;
            tileBase += tilesX * tilesY;
            pixBase += c.pixels;
        }
        const uint32_t chunkTiles = tileBase;
        const uint32_t keyBits = 24 + bits_for(chunkTiles);
        const uint32_t lastPartition = count * lrt::project_partitions(n) - 1;
        std::vector<lrt::ViewParams> hostViews(count);
        std::vector<FrameParams> hostFrames(count);
        for (uint32_t k = 0; k < count; ++k) {
            hostViews[k] = cv[k].v;
            hostFrames[k] = cv[k].f;
        }
        LRT_CUDA(r, cudaMemcpyAsync(devViews, hostViews.data(), count * sizeof(lrt::ViewParams), cudaMemcpyHostToDevice,
                                    stream),
                 "view parameters");
        LRT_CUDA(r, cudaMemcpyAsync(r->trainBatchFrames.ptr, hostFrames.data(), count * sizeof(FrameParams),
                                    cudaMemcpyHostToDevice, stream),
                 "frame parameters");

        // --- forward: project, sort, ranges, blend (drawn again if the pairs outgrew their buffer) ---
        const uint64_t* sorted = nullptr;
        const uint32_t* emit = nullptr;
        uint32_t pairs = 0;
        for (int attempt = 0; attempt < 2; ++attempt) {
            const uint32_t cap = r->trainBatchPairCap;
            LRT_CUDA(r, ensure(r->pairs, size_t{cap} * 8), "pairs");
            LRT_CUDA(r, ensure(r->pairsAlt, size_t{cap} * 8), "pairs");
            LRT_CUDA(r, ensure(r->pairValues, size_t{cap} * 4), "pair values");
            LRT_CUDA(r, ensure(r->pairValuesAlt, size_t{cap} * 4), "pair values");
            LRT_CUDA(r, ensure(r->sortScratch, lrt::sort_scratch_bytes(cap, keyBits)), "sort scratch");
            LRT_CUDA(r, cudaMemsetAsync(counters, 0, 16, stream), "counters");
            LRT_CUDA(r, cudaMemsetAsync(r->scanScratch.ptr, 0, statusBytes, stream), "projection scratch");
            LRT_CUDA(r, cudaMemsetAsync(queue, 0, 4, stream), "queue");
            uint64_t* pairBuf = static_cast<uint64_t*>(r->pairs.ptr);
            uint32_t* valueBuf = static_cast<uint32_t*>(r->pairValues.ptr);
            uint32_t partitionBase = 0;
            for (uint32_t k = 0; k < count; ++k) {
                LRT_CUDA(r,
                         lrt::launch_project_emit_train(
                             cv[k].f, means, logScales, quats, logits, sh, static_cast<ProjRecord*>(r->proj.ptr),
                             nullptr, static_cast<uint32_t*>(r->touched.ptr), nullptr,
                             static_cast<uint32_t*>(r->trainOffsets.ptr) + size_t{k} * n, counters, status,
                             tickets + k, partitionBase, lastPartition, slotBits, pairBuf, valueBuf, nullptr, cap,
                             stream),
                         "project");
                partitionBase += lrt::project_partitions(n);
            }
            bool inAlt = false;
            LRT_CUDA(r,
                     lrt::launch_sort_u64(pairBuf, static_cast<uint64_t*>(r->pairsAlt.ptr), valueBuf,
                                          static_cast<uint32_t*>(r->pairValuesAlt.ptr), counters + 1, cap, slotBits,
                                          keyBits, r->sortScratch.ptr, err, &inAlt, stream),
                     "pair sort");
            sorted = inAlt ? static_cast<uint64_t*>(r->pairsAlt.ptr) : pairBuf;
            emit = inAlt ? static_cast<uint32_t*>(r->pairValuesAlt.ptr) : valueBuf;
            LRT_CUDA(r,
                     lrt::launch_ranges(sorted, counters + 1, cap, 24 + slotBits, static_cast<uint2*>(r->ranges.ptr),
                                        chunkTiles, stream),
                     "ranges");
            LRT_CUDA(r,
                     lrt::launch_blend_batch_train(bp, devViews, count, static_cast<uint2*>(r->ranges.ptr), sorted,
                                                   static_cast<ProjRecord*>(r->proj.ptr), chunkTiles, queue, err,
                                                   static_cast<uint32_t>(numSMs) * kTrainBlendBlocksPerSM, stream),
                     "blend");
            LRT_CUDA(r, cudaMemcpyAsync(r->hostCounters, counters, 16, cudaMemcpyDeviceToHost, stream), "readback");
            LRT_CUDA(r, cudaStreamSynchronize(stream), "chunk");
            pairs = r->hostCounters[1];
            const uint32_t statusBits = r->hostCounters[2];
            if (statusBits & lrt::kErrTooManyPairs) return fail(r, LRT_UNSUPPORTED, "more than 2^32 pairs in a chunk");
            if (statusBits & lrt::kErrTimeout) return fail(r, LRT_TIMEOUT, "a bounded device wait gave up");
            if (pairs <= cap) break;
            r->trainBatchPairCap = grow(r->trainBatchPairCap, pairs);   // draw the chunk again with room
            if (attempt == 1) return fail(r, LRT_OVERFLOW, "pair capacity exceeded");
        }
        totalPairs += pairs;

        // --- the loss, and its gradient with respect to each view's colour ---
        for (uint32_t k = 0; k < count; ++k) {
            const lrt_train_view& vw = views[c0 + k];
            float* loss = vw.loss != nullptr ? static_cast<float*>(vw.loss) : static_cast<float*>(r->trainBatchLoss.ptr) + k;
            LRT_CUDA(r,
                     lrt::launch_l1_loss(static_cast<const float4*>(vw.colour), static_cast<const float*>(vw.target),
                                         cv[k].pixels, static_cast<float*>(r->lossScratch.ptr), loss, stream),
                     "loss");
            LRT_CUDA(r,
                     lrt::launch_l1_grad(static_cast<const float4*>(vw.colour), static_cast<const float*>(vw.target),
                                         cv[k].pixels, nullptr,
                                         static_cast<float4*>(r->trainBatchGrad.ptr) + cv[k].pixBase, stream),
                     "loss gradient");
        }

        // --- backward: per-pair partials over the chunk's tiles, then per splat over the chunk's views ---
        LRT_CUDA(r, ensure(r->partials, size_t{std::max(pairs, 1u)} * 48), "pair partials");
        LRT_CUDA(r,
                 lrt::launch_blend_backward_batch(bp, devViews, count, static_cast<uint2*>(r->ranges.ptr), sorted, emit,
                                                  static_cast<ProjRecord*>(r->proj.ptr), chunkTiles,
                                                  static_cast<float*>(r->partials.ptr), stream),
                 "blend backward");
        LRT_CUDA(r,
                 lrt::launch_splat_backward_views(static_cast<const FrameParams*>(r->trainBatchFrames.ptr), count, n,
                                                  means, logScales, quats, logits, sh,
                                                  static_cast<uint32_t*>(r->touched.ptr),
                                                  static_cast<uint32_t*>(r->trainOffsets.ptr),
                                                  static_cast<float*>(r->partials.ptr), pairs,
                                                  static_cast<float*>(grads->means),
                                                  static_cast<float*>(grads->log_scales),
                                                  static_cast<float*>(grads->quats),
                                                  static_cast<float*>(grads->opacity_logits),
                                                  static_cast<float*>(grads->sh), c0 > 0, stream),
                 "projection backward");
    }
    LRT_CUDA(r, cudaEventRecord(r->ev[7], stream), "event");
    LRT_CUDA(r, cudaEventRecord(r->frameDone, stream), "event");
    r->frameDoneSet = true;
    LRT_CUDA(r, cudaStreamSynchronize(stream), "batch");
    if (stats != nullptr) {
        stats->views = nViews;
        stats->splats = n;
        stats->pairs = static_cast<uint32_t>(std::min<uint64_t>(totalPairs, 0xFFFFFFFFull));
        stats->chunks = chunks;
        stats->views_per_chunk = perChunk;
        stats->blend_blocks_per_sm = kTrainBlendBlocksPerSM;
        stats->device_ms = event_ms(r->ev[6], r->ev[7]);
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return LRT_OK;
}
