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
//   emit indices -> per-splat backward over the chunk's views: each splat's
//   gradients summed view after view (from zero in the batch's first chunk,
//   from the buffers' values in later ones) and written once.
// Each view's pixels, and each view's gradient contribution, are the same
// bits as a single-view training step of that view: within a tile the pairs
// keep the single view's order, and a splat's pairs are contiguous at their
// emit indices as in a single view.
//
// The whole step is enqueued without a host wait between chunks: every
// chunk has its own counter words, the pair buffers are sized from the
// largest chunk seen for this shape, and the counters of all chunks are read
// back once at the end. A chunk that outgrew the pair buffer (only possible
// when the cameras changed) makes the step run again with room. The view and
// frame parameters of every chunk live in device memory, staged in pinned
// memory, so no kernel argument depends on the cameras: the first steps of a
// shape time a few chunk sizes and blend grid sizes and keep the fastest, the
// next one is captured into a CUDA graph, and later ones replay it with the
// new cameras (a new graph when a buffer, a pointer or the shape changes).
#include "rast_handle.h"

#include <algorithm>
#include <chrono>
#include <cstring>

namespace {

constexpr uint32_t kDefaultChunkViews = 16;
constexpr uint32_t kDefaultBlocksPerSM = 4;
constexpr uint32_t kBackwardViews = 16;    // views one per-splat backward launch takes

uint64_t tb_mix(uint64_t h, uint64_t v) {
    h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    return h;
}

// Grows a buffer and, when it moves, invalidates the captured step.
cudaError_t ensure_tb(lrt_rast* r, DeviceBuffer& b, size_t bytes) {
    if (b.bytes >= bytes && b.ptr != nullptr) return cudaSuccess;
    r->trainBatch.generation += 1;
    return ensure(b, bytes);
}

// Where each view sits for one chunk size: its chunk, its frame and view
// parameters (tiles and records numbered within the chunk), its pixels.
struct Layout {
    uint32_t perChunk = 0, chunks = 0;
    std::vector<uint32_t> chunkTiles;
    std::vector<FrameParams> frames;          // one per view
    std::vector<lrt::ViewParams> viewParams;  // one per view
    std::vector<size_t> pixBase;              // each view's first pixel in its chunk's pixel buffers
    size_t maxPixels = 0;
    uint32_t maxTiles = 0;
};

Layout make_layout(lrt_rast* r, const lrt_train_view* views, uint32_t nViews, const lrt_render_settings* s,
                   const CloudDesc& cloud, uint32_t perChunk) {
    Layout L;
    L.perChunk = perChunk;
    L.chunks = (nViews + perChunk - 1) / perChunk;
    L.frames.resize(nViews);
    L.viewParams.resize(nViews);
    L.pixBase.resize(nViews);
    const uint32_t n = cloud.count;
    for (uint32_t c = 0; c < L.chunks; ++c) {
        uint32_t tileBase = 0;
        size_t pix = 0;
        for (uint32_t v = c * perChunk; v < std::min(nViews, (c + 1) * perChunk); ++v) {
            const uint32_t k = v - c * perChunk;
            const lrt_train_view& vw = views[v];
            lrt_render_settings sv = *s;
            sv.width = vw.width;
            sv.height = vw.height;
            const uint32_t tilesX = (vw.width + lrt::kTile - 1) / lrt::kTile;
            const uint32_t tilesY = (vw.height + lrt::kTile - 1) / lrt::kTile;
            FrameParams f = frame_params(&vw.projection, &sv, cloud, tilesX, tilesY, 0);
            f.tileBase = tileBase;
            f.recordBase = k * n;
            f.writeDebug = 0;
            L.frames[v] = f;
            lrt::ViewParams& p = L.viewParams[v];
            p = lrt::ViewParams{};
            p.width = vw.width;
            p.height = vw.height;
            p.tilesX = tilesX;
            p.tileBase = tileBase;
            p.recordBase = k * n;
            p.colour = static_cast<float4*>(vw.colour);
            p.depth = static_cast<float*>(vw.depth);
            p.pixState = static_cast<float4*>(r->pixState.ptr) + pix;
            p.pixLast = static_cast<uint32_t*>(r->pixLast.ptr) + pix;
            p.gradColour = static_cast<const float4*>(r->trainBatchGrad.ptr) + pix;
            L.pixBase[v] = pix;
            tileBase += tilesX * tilesY;
            pix += size_t{vw.width} * vw.height;
        }
        L.chunkTiles.push_back(tileBase);
        L.maxTiles = std::max(L.maxTiles, tileBase);
        L.maxPixels = std::max(L.maxPixels, pix);
    }
    return L;
}

// The per-pixel pointers of the views depend on the pixel buffers, which a
// larger chunk can move: set them once the buffers are in place.
void place_pixels(lrt_rast* r, Layout& L) {
    for (size_t v = 0; v < L.viewParams.size(); ++v) {
        L.viewParams[v].pixState = static_cast<float4*>(r->pixState.ptr) + L.pixBase[v];
        L.viewParams[v].pixLast = static_cast<uint32_t*>(r->pixLast.ptr) + L.pixBase[v];
        L.viewParams[v].gradColour = static_cast<const float4*>(r->trainBatchGrad.ptr) + L.pixBase[v];
    }
}

struct StepArgs {
    const lrt_train_params* params;
    const lrt_train_view* views;
    uint32_t nViews;
    const lrt_render_settings* s;
    const lrt_train_grads* grads;
    uint32_t numSMs;
};

// The buffers of a step with this layout, for `cap` pairs a chunk.
int reserve_step(lrt_rast* r, const StepArgs& a, const Layout& L, uint32_t cap) {
    auto& T = r->trainBatch;
    const uint32_t n = a.params->count;
    const uint64_t slots = uint64_t{L.perChunk} * n;
    const uint64_t partitions = uint64_t{L.perChunk} * lrt::project_partitions(n);
    const size_t statusBytes = lrt::project_status_bytes(static_cast<uint32_t>(partitions)) + size_t{L.perChunk} * 4;
    const uint32_t keyBits = 24 + bits_for(L.maxTiles);
    LRT_CUDA(r, ensure_tb(r, r->proj, slots * sizeof(ProjRecord)), "splat records");
    LRT_CUDA(r, ensure_tb(r, r->touched, slots * 4), "touched counts");
    LRT_CUDA(r, ensure_tb(r, r->pairOffsets, slots * 4), "pair offsets");
    LRT_CUDA(r, ensure_tb(r, r->pixState, L.maxPixels * 16), "pixel state");
    LRT_CUDA(r, ensure_tb(r, r->pixLast, L.maxPixels * 4), "pixel state");
    LRT_CUDA(r, ensure_tb(r, r->trainBatchGrad, L.maxPixels * 16), "colour gradients");
    const size_t paramBytes = size_t{a.nViews} * (sizeof(lrt::ViewParams) + sizeof(FrameParams));
    LRT_CUDA(r, ensure_tb(r, r->trainBatchViews, paramBytes + 16 + size_t{L.chunks} * 4), "view parameters");
    LRT_CUDA(r, ensure_tb(r, r->trainBatchLoss, size_t{a.nViews} * 4 + 16), "losses");
    LRT_CUDA(r, ensure_tb(r, r->lossScratch, lrt::l1_scratch_bytes()), "loss scratch");
    LRT_CUDA(r, ensure_tb(r, r->scanScratch, std::max<size_t>(statusBytes, 16)), "projection scratch");
    LRT_CUDA(r, ensure_tb(r, r->ranges, size_t{L.maxTiles} * 8), "tile ranges");
    LRT_CUDA(r, ensure_tb(r, r->pairs, size_t{cap} * 8), "pairs");
    LRT_CUDA(r, ensure_tb(r, r->pairsAlt, size_t{cap} * 8), "pairs");
    LRT_CUDA(r, ensure_tb(r, r->pairValues, size_t{cap} * 4), "pair values");
    LRT_CUDA(r, ensure_tb(r, r->pairValuesAlt, size_t{cap} * 4), "pair values");
    LRT_CUDA(r, ensure_tb(r, r->sortScratch, lrt::sort_scratch_bytes(cap, keyBits)), "sort scratch");
    LRT_CUDA(r, ensure_tb(r, r->partials, size_t{cap} * 48), "pair partials");
    LRT_CUDA(r, ensure_tb(r, T.counters, size_t{L.chunks} * 16), "chunk counters");
    if (T.hostParamsBytes < paramBytes) {
        if (T.hostParams != nullptr) cudaFreeHost(T.hostParams);
        T.hostParams = nullptr;
        T.hostParamsBytes = 0;
        LRT_CUDA(r, cudaMallocHost(&T.hostParams, paramBytes), "pinned parameters");
        T.hostParamsBytes = paramBytes;
        T.generation += 1;
    }
    if (T.hostCounterChunks < L.chunks) {
        if (T.hostCounters != nullptr) cudaFreeHost(T.hostCounters);
        T.hostCounters = nullptr;
        T.hostCounterChunks = 0;
        LRT_CUDA(r, cudaMallocHost(&T.hostCounters, size_t{L.chunks} * 16), "pinned counters");
        T.hostCounterChunks = L.chunks;
        T.generation += 1;
    }
    return LRT_OK;
}

// The cameras of this call into the pinned staging buffer (view parameters
// for every view, then frame parameters for every view).
void stage_params(lrt_rast* r, const Layout& L) {
    auto& T = r->trainBatch;
    const size_t nv = L.viewParams.size();
    std::memcpy(T.hostParams, L.viewParams.data(), nv * sizeof(lrt::ViewParams));
    std::memcpy(static_cast<char*>(T.hostParams) + nv * sizeof(lrt::ViewParams), L.frames.data(),
                nv * sizeof(FrameParams));
}

// The whole step on the batch stream, from the staged parameters' upload to
// the counters' readback.
int enqueue_step(lrt_rast* r, const StepArgs& a, const Layout& L, uint32_t cap, uint32_t blocksPerSM) {
    auto& T = r->trainBatch;
    cudaStream_t st = T.stream;
    const uint32_t n = a.params->count;
    const size_t nv = a.nViews;
    const size_t paramBytes = nv * (sizeof(lrt::ViewParams) + sizeof(FrameParams));
    LRT_CUDA(r, cudaMemcpyAsync(r->trainBatchViews.ptr, T.hostParams, paramBytes, cudaMemcpyHostToDevice, st),
             "view parameters");
    const lrt::ViewParams* devViews = static_cast<const lrt::ViewParams*>(r->trainBatchViews.ptr);
    const FrameParams* devFrames =
        reinterpret_cast<const FrameParams*>(static_cast<const char*>(r->trainBatchViews.ptr) + nv * sizeof(lrt::ViewParams));
    uint32_t* queues = reinterpret_cast<uint32_t*>(static_cast<char*>(r->trainBatchViews.ptr) + paramBytes + 16);
    const uint32_t slotBits = bits_for(n);
    const uint64_t partitions = uint64_t{L.perChunk} * lrt::project_partitions(n);
    const size_t statusBytes = lrt::project_status_bytes(static_cast<uint32_t>(partitions)) + size_t{L.perChunk} * 4;
    uint64_t* status = static_cast<uint64_t*>(r->scanScratch.ptr);
    uint32_t* tickets = reinterpret_cast<uint32_t*>(static_cast<char*>(r->scanScratch.ptr) +
                                                    lrt::project_status_bytes(static_cast<uint32_t>(partitions)));
    BlendParams bp{};
    bp.slotBits = slotBits;
    bp.tileShift = 24 + slotBits;
    bp.depthMode = a.s->depth_mode;
    bp.linearise = a.s->linearise ? 1u : 0u;
    bp.depthThreshold = a.s->depth_threshold;
    for (int k = 0; k < 4; ++k) bp.bg[k] = a.s->background[k];
    const auto* p = a.params;
    const float* means = static_cast<const float*>(p->means);
    const float* logScales = static_cast<const float*>(p->log_scales);
    const float* quats = static_cast<const float*>(p->quats);
    const float* logits = static_cast<const float*>(p->opacity_logits);
    const uint16_t* sh = static_cast<const uint16_t*>(p->sh);
    uint32_t* allCounters = static_cast<uint32_t*>(T.counters.ptr);
    LRT_CUDA(r, cudaMemsetAsync(allCounters, 0, size_t{L.chunks} * 16, st), "counters");
    LRT_CUDA(r, cudaMemsetAsync(queues, 0, size_t{L.chunks} * 4, st), "queues");
    for (uint32_t c = 0; c < L.chunks; ++c) {
        const uint32_t v0 = c * L.perChunk, v1 = std::min(a.nViews, v0 + L.perChunk), count = v1 - v0;
        const uint32_t chunkTiles = L.chunkTiles[c];
        const uint32_t keyBits = 24 + bits_for(chunkTiles);
        uint32_t* counters = allCounters + 4 * c;
        uint32_t* err = counters + 2;
        // --- forward: project, sort, ranges, blend ---
        LRT_CUDA(r, cudaMemsetAsync(r->scanScratch.ptr, 0, statusBytes, st), "projection scratch");
        uint64_t* pairBuf = static_cast<uint64_t*>(r->pairs.ptr);
        uint32_t* valueBuf = static_cast<uint32_t*>(r->pairValues.ptr);
        const uint32_t lastPartition = count * lrt::project_partitions(n) - 1;
        uint32_t partitionBase = 0;
        for (uint32_t v = v0; v < v1; ++v) {
            const uint32_t k = v - v0;
            LRT_CUDA(r,
                     lrt::launch_project_emit_train(
                         L.frames[v], means, logScales, quats, logits, sh, static_cast<ProjRecord*>(r->proj.ptr),
                         nullptr, static_cast<uint32_t*>(r->touched.ptr), nullptr,
                         static_cast<uint32_t*>(r->pairOffsets.ptr) + size_t{k} * n, counters, status, tickets + k,
                         partitionBase, lastPartition, slotBits, pairBuf, valueBuf, nullptr, cap, st, devFrames + v),
                     "project");
            partitionBase += lrt::project_partitions(n);
        }
        bool inAlt = false;
        LRT_CUDA(r,
                 lrt::launch_sort_u64(pairBuf, static_cast<uint64_t*>(r->pairsAlt.ptr), valueBuf,
                                      static_cast<uint32_t*>(r->pairValuesAlt.ptr), counters + 1, cap, slotBits,
                                      keyBits, r->sortScratch.ptr, err, &inAlt, st),
                 "pair sort");
        const uint64_t* sorted = inAlt ? static_cast<uint64_t*>(r->pairsAlt.ptr) : pairBuf;
        const uint32_t* emit = inAlt ? static_cast<uint32_t*>(r->pairValuesAlt.ptr) : valueBuf;
        LRT_CUDA(r,
                 lrt::launch_ranges(sorted, counters + 1, cap, 24 + slotBits, static_cast<uint2*>(r->ranges.ptr),
                                    chunkTiles, st),
                 "ranges");
        LRT_CUDA(r,
                 lrt::launch_blend_batch_train(bp, devViews + v0, count, static_cast<uint2*>(r->ranges.ptr), sorted,
                                               static_cast<ProjRecord*>(r->proj.ptr), chunkTiles, queues + c, err,
                                               a.numSMs * blocksPerSM, st),
                 "blend");
        // --- the loss, and its gradient with respect to each view's colour ---
        for (uint32_t v = v0; v < v1; ++v) {
            const lrt_train_view& vw = a.views[v];
            const uint32_t pixels = vw.width * vw.height;
            float* loss = vw.loss != nullptr ? static_cast<float*>(vw.loss) : static_cast<float*>(r->trainBatchLoss.ptr) + v;
            LRT_CUDA(r,
                     lrt::launch_l1_loss(static_cast<const float4*>(vw.colour), static_cast<const float*>(vw.target),
                                         pixels, static_cast<float*>(r->lossScratch.ptr), loss, st),
                     "loss");
            LRT_CUDA(r,
                     lrt::launch_l1_grad(static_cast<const float4*>(vw.colour), static_cast<const float*>(vw.target),
                                         pixels, nullptr, static_cast<float4*>(r->trainBatchGrad.ptr) + L.pixBase[v],
                                         st),
                     "loss gradient");
        }
        // --- backward: per-pair partials over the chunk's tiles, then per splat over its views ---
        LRT_CUDA(r,
                 lrt::launch_blend_backward_batch(bp, devViews + v0, count, static_cast<uint2*>(r->ranges.ptr), sorted,
                                                  emit, static_cast<ProjRecord*>(r->proj.ptr), chunkTiles,
                                                  static_cast<float*>(r->partials.ptr), st),
                 "blend backward");
        for (uint32_t b0 = 0; b0 < count; b0 += kBackwardViews) {
            const uint32_t bn = std::min(kBackwardViews, count - b0);
            LRT_CUDA(r,
                     lrt::launch_splat_backward_views(
                         devFrames + v0 + b0, bn, n, means, logScales, quats, logits, sh,
                         static_cast<uint32_t*>(r->touched.ptr) + size_t{b0} * n,
                         static_cast<uint32_t*>(r->pairOffsets.ptr) + size_t{b0} * n,
                         static_cast<float*>(r->partials.ptr), cap, static_cast<float*>(a.grads->means),
                         static_cast<float*>(a.grads->log_scales), static_cast<float*>(a.grads->quats),
                         static_cast<float*>(a.grads->opacity_logits), static_cast<float*>(a.grads->sh),
                         v0 + b0 > 0, st),
                     "projection backward");
        }
    }
    LRT_CUDA(r, cudaMemcpyAsync(T.hostCounters, allCounters, size_t{L.chunks} * 16, cudaMemcpyDeviceToHost, st),
             "counters");
    return LRT_OK;
}

// What a captured step depends on besides the buffers (their moves bump the
// generation): the shape, the chunking, the pointers its launches take.
uint64_t step_key(const lrt_rast* r, const StepArgs& a, const Layout& L, uint32_t cap, uint32_t blocksPerSM) {
    uint64_t k = tb_mix(0, a.params->count);
    k = tb_mix(k, a.nViews);
    k = tb_mix(tb_mix(k, L.perChunk), blocksPerSM);
    k = tb_mix(k, cap);
    for (const void* q : {a.params->means, a.params->log_scales, a.params->quats, a.params->opacity_logits,
                          a.params->sh, static_cast<const void*>(a.grads->means), static_cast<const void*>(a.grads->log_scales),
                          static_cast<const void*>(a.grads->quats), static_cast<const void*>(a.grads->opacity_logits),
                          static_cast<const void*>(a.grads->sh)})
        k = tb_mix(k, reinterpret_cast<uintptr_t>(q));
    for (uint32_t v = 0; v < a.nViews; ++v) {
        const lrt_train_view& vw = a.views[v];
        k = tb_mix(tb_mix(k, vw.width), vw.height);
        for (const void* q : {static_cast<const void*>(vw.colour), static_cast<const void*>(vw.depth), vw.target,
                              static_cast<const void*>(vw.loss)})
            k = tb_mix(k, reinterpret_cast<uintptr_t>(q));
    }
    // The handle's buffers, which single-view steps and frames share and can
    // move between batches.
    for (const DeviceBuffer* b : {&r->proj, &r->touched, &r->pairOffsets, &r->pixState, &r->pixLast,
                                  &r->trainBatchGrad, &r->trainBatchViews, &r->trainBatchLoss, &r->lossScratch,
                                  &r->scanScratch, &r->ranges, &r->pairs, &r->pairsAlt, &r->pairValues,
                                  &r->pairValuesAlt, &r->sortScratch, &r->partials, &r->trainBatch.counters})
        k = tb_mix(k, reinterpret_cast<uintptr_t>(b->ptr));
    k = tb_mix(tb_mix(k, reinterpret_cast<uintptr_t>(r->trainBatch.hostParams)),
               reinterpret_cast<uintptr_t>(r->trainBatch.hostCounters));
    const lrt_render_settings* s = a.s;
    k = tb_mix(k, (uint64_t{s->antialias} << 1) ^ (uint64_t{s->max_sh_degree} << 3) ^ (uint64_t{s->linearise} << 7) ^
                      (uint64_t{s->depth_mode} << 9));
    uint32_t bits[5];
    std::memcpy(bits, s->background, 16);
    std::memcpy(bits + 4, &s->depth_threshold, 4);
    for (uint32_t b : bits) k = tb_mix(k, b);
    return k;
}

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
        if (views[v].width > lrt::kMaxFrameSide || views[v].height > lrt::kMaxFrameSide)
            return fail(r, LRT_UNSUPPORTED, "a view side above 2^19 pixels");
        if (views[v].colour == nullptr || views[v].depth == nullptr || views[v].target == nullptr)
            return fail(r, LRT_INVALID_ARGUMENT, "a view without its images or target");
    }
    if (stats != nullptr) std::memset(stats, 0, sizeof(*stats));
    if (nViews == 0) return LRT_OK;

    DeviceScope scope(r->device);
    auto& T = r->trainBatch;
    cudaStream_t caller = static_cast<cudaStream_t>(streamPtr);
    if (T.stream == nullptr) {
        LRT_CUDA(r, cudaStreamCreateWithFlags(&T.stream, cudaStreamNonBlocking), "training batch stream");
        for (cudaEvent_t* e : {&T.in, &T.out, &T.start, &T.end}) LRT_CUDA(r, cudaEventCreate(e), "batch event");
    }
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
    const StepArgs args{params, views, nViews, s, grads, static_cast<uint32_t>(numSMs)};

    // The shape (what tuning is kept for): splat count and the views' sizes.
    uint64_t shapeKey = tb_mix(0, n);
    for (uint32_t v = 0; v < nViews; ++v) shapeKey = tb_mix(tb_mix(shapeKey, views[v].width), views[v].height);
    uint32_t perChunk = std::min(nViews, kDefaultChunkViews), blocksPerSM = kDefaultBlocksPerSM;
    bool tuning = true;
    for (const auto& e : T.tuned)
        if (e.first == shapeKey) {
            perChunk = e.second.first;
            blocksPerSM = e.second.second;
            tuning = false;
        }
    if (T.fixedChunk != 0) {
        perChunk = std::min(nViews, T.fixedChunk);
        blocksPerSM = T.fixedBlocks != 0 ? T.fixedBlocks : kDefaultBlocksPerSM;
        tuning = false;
    }

    auto check_layout = [&](uint32_t chunk, Layout& L) -> int {
        L = make_layout(r, views, nViews, s, cloud, chunk);
        if (uint64_t{chunk} * n > 0xFFFFFFFFull) return fail(r, LRT_UNSUPPORTED, "a chunk's records pass 2^32");
        if (bits_for(n) + 24 + bits_for(L.maxTiles) > 64)
            return fail(r, LRT_UNSUPPORTED, "splat slots and a chunk's tiles do not fit one 64-bit pair word");
        return LRT_OK;
    };
    // Counters of the last run: the largest chunk's pairs and every status bit.
    auto read_counters = [&](const Layout& L, uint32_t* worst, uint32_t* statusBits, uint64_t* total) {
        *worst = 0;
        *statusBits = 0;
        *total = 0;
        for (uint32_t c = 0; c < L.chunks; ++c) {
            *worst = std::max(*worst, T.hostCounters[4 * c + 1]);
            *statusBits |= T.hostCounters[4 * c + 2];
            *total += T.hostCounters[4 * c + 1];
        }
    };
    uint64_t totalPairs = 0;
    // One eager run, drawn again with room while a chunk outgrows the pairs.
    auto eager = [&](Layout& L, uint32_t bps, float* ms) -> int {
        for (int attempt = 0; attempt < 3; ++attempt) {
            if (r->trainBatchPairCap == 0)
                r->trainBatchPairCap = std::max<uint32_t>(
                    1024, static_cast<uint32_t>(std::min<uint64_t>(uint64_t{L.perChunk} * n * 4, 0xFFFFFFFFull)));
            const uint32_t cap = r->trainBatchPairCap;
            int code = reserve_step(r, args, L, cap);
            if (code != LRT_OK) return code;
            place_pixels(r, L);
            stage_params(r, L);
            LRT_CUDA(r, cudaEventRecord(T.start, T.stream), "event");
            code = enqueue_step(r, args, L, cap, bps);
            if (code != LRT_OK) return code;
            LRT_CUDA(r, cudaEventRecord(T.end, T.stream), "event");
            LRT_CUDA(r, cudaStreamSynchronize(T.stream), "training batch");
            LRT_CUDA(r, cudaEventElapsedTime(ms, T.start, T.end), "event");
            uint32_t worst = 0, statusBits = 0;
            read_counters(L, &worst, &statusBits, &totalPairs);
            if (statusBits & lrt::kErrTooManyPairs) return fail(r, LRT_UNSUPPORTED, "more than 2^32 pairs in a chunk");
            if (statusBits & lrt::kErrTimeout) return fail(r, LRT_TIMEOUT, "a bounded device wait gave up");
            if (worst <= cap) return LRT_OK;
            r->trainBatchPairCap = grow(r->trainBatchPairCap, worst);   // run the step again with room
        }
        return fail(r, LRT_OVERFLOW, "pair capacity exceeded");
    };

    LRT_CUDA(r, cudaEventRecord(T.in, caller), "event");
    LRT_CUDA(r, cudaStreamWaitEvent(T.stream, T.in, 0), "event");
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(T.stream, r->frameDone, 0), "frame order");
    Layout L;
    bool replayed = false;
    float deviceMs = 0.0f;
    if (tuning) {
        // Views per chunk x blend blocks per SM, the fastest of one timed
        // run each (after a run that sizes the buffers). Every run is a whole
        // step, so the gradients of the last one stand whichever wins.
        std::vector<uint32_t> sizes;
        for (uint32_t c : {8u, 16u, 32u, nViews})
            if (c <= nViews && std::find(sizes.begin(), sizes.end(), c) == sizes.end()) sizes.push_back(c);
        if (sizes.empty()) sizes.push_back(nViews);
        float best = 3.4e38f;
        for (uint32_t c : sizes) {
            int code = check_layout(c, L);
            if (code != LRT_OK) return code;
            for (uint32_t bps : {4u, 8u}) {
                float ms = 0.0f;
                code = eager(L, bps, &ms);   // sizes the buffers
                if (code != LRT_OK) return code;
                code = eager(L, bps, &ms);
                if (code != LRT_OK) return code;
                if (ms < best) {
                    best = ms;
                    perChunk = c;
                    blocksPerSM = bps;
                }
            }
        }
        T.tuned.push_back({shapeKey, {perChunk, blocksPerSM}});
        int code = check_layout(perChunk, L);
        if (code != LRT_OK) return code;
        code = eager(L, blocksPerSM, &deviceMs);   // the step itself, with the choice
        if (code != LRT_OK) return code;
    } else {
        int code = check_layout(perChunk, L);
        if (code != LRT_OK) return code;
        if (r->trainBatchPairCap == 0) {   // a fixed chunking's first step sizes the buffers
            code = eager(L, blocksPerSM, &deviceMs);
            if (code != LRT_OK) return code;
        }
        const uint32_t cap = r->trainBatchPairCap;
        code = reserve_step(r, args, L, cap);
        if (code != LRT_OK) return code;
        place_pixels(r, L);
        stage_params(r, L);
        const uint64_t key = step_key(r, args, L, cap, blocksPerSM);
        const bool haveGraph = T.graph != nullptr && T.graphKey == key && T.graphGeneration == T.generation;
        if (!haveGraph && !T.graphFailed) {
            if (T.graph != nullptr) {
                cudaGraphExecDestroy(T.graph);
                T.graph = nullptr;
            }
            cudaGraph_t graph = nullptr;
            bool ok = cudaStreamBeginCapture(T.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                code = enqueue_step(r, args, L, cap, blocksPerSM);
                ok = cudaStreamEndCapture(T.stream, &graph) == cudaSuccess && code == LRT_OK;
            }
            if (ok) ok = cudaGraphInstantiate(&T.graph, graph, 0) == cudaSuccess;
            if (graph != nullptr) cudaGraphDestroy(graph);
            cudaGetLastError();
            if (ok) {
                T.graphKey = key;
                T.graphGeneration = T.generation;
            } else {
                T.graph = nullptr;
                T.graphFailed = true;   // keep running eagerly
                r->error.clear();
            }
        }
        if (T.graph != nullptr && T.graphKey == key && T.graphGeneration == T.generation) {
            LRT_CUDA(r, cudaEventRecord(T.start, T.stream), "event");
            LRT_CUDA(r, cudaGraphLaunch(T.graph, T.stream), "graph launch");
            LRT_CUDA(r, cudaEventRecord(T.end, T.stream), "event");
            LRT_CUDA(r, cudaStreamSynchronize(T.stream), "training batch");
            LRT_CUDA(r, cudaEventElapsedTime(&deviceMs, T.start, T.end), "event");
            uint32_t worst = 0, statusBits = 0;
            read_counters(L, &worst, &statusBits, &totalPairs);
            if (statusBits & lrt::kErrTooManyPairs) return fail(r, LRT_UNSUPPORTED, "more than 2^32 pairs in a chunk");
            if (statusBits & lrt::kErrTimeout) return fail(r, LRT_TIMEOUT, "a bounded device wait gave up");
            replayed = worst <= cap;
            if (!replayed) r->trainBatchPairCap = grow(r->trainBatchPairCap, worst);
        }
        if (!replayed) {
            code = eager(L, blocksPerSM, &deviceMs);
            if (code != LRT_OK) return code;
        }
    }
    LRT_CUDA(r, cudaEventRecord(T.out, T.stream), "event");
    LRT_CUDA(r, cudaStreamWaitEvent(caller, T.out, 0), "event");
    LRT_CUDA(r, cudaEventRecord(r->frameDone, T.stream), "event");
    r->frameDoneSet = true;
    if (stats != nullptr) {
        stats->views = nViews;
        stats->splats = n;
        stats->pairs = static_cast<uint32_t>(std::min<uint64_t>(totalPairs, 0xFFFFFFFFull));
        stats->chunks = L.chunks;
        stats->views_per_chunk = perChunk;
        stats->blend_blocks_per_sm = blocksPerSM;
        stats->graph_replayed = replayed ? 1u : 0u;
        stats->device_ms = deviceMs;
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return LRT_OK;
}

extern "C" int lrt_rast_debug_train_chunking(lrt_rast* r, uint32_t views_per_chunk, uint32_t blocks_per_sm) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    r->trainBatch.fixedChunk = views_per_chunk;
    r->trainBatch.fixedBlocks = blocks_per_sm;
    return LRT_OK;
}
