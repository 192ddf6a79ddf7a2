// The levels of detail's C-ABI (include/lrt_raster.h): LodBuilder::build and
// CutSelector::select (modules/lod/src/Lod.cpp:86-547) over lod.cu's kernels.
//
// A build waits twice: once for the bounds and every level's group count
// (which size the levels' buffers), once at its end, when the group counts
// the compactions found are checked against them. The reference waits and
// reads once per level and once per stage. A select runs one cut (two
// kernels) per instance and waits once for all their counts; a cut whose drawn count
// passes its cloud's capacity (possible only if the float size test were
// not monotone down the tree) is grown and run again.
#include "rast_handle.h"

#include <cstring>

#include "lookback.cuh"

using lrt::kLodLevels;
using lrt::kLodMomentsHead;
using lrt::LodCutParams;
using lrt::LodGlobals;
using lrt::LodSplatArrays;

struct lrt_lod {
    int device = 0;
    uint32_t count = 0, restPerColour = 0, shWords = 0;
    uint32_t coarsest = 0, finest = 0, levels = 0, merged = 0, chunkSplats = 0;
    float boundsLo[3] = {0, 0, 0}, boundsHi[3] = {0, 0, 0}, extent = 0.0f;
    uint32_t levelBase[kLodLevels + 2] = {};           // first merged Gaussian of each stored level; [levels] = merged
    // The store (Morton order) and the merged Gaussians (coarsest level
    // first) with their cells and the finest groups' starts, each set carved
    // from one allocation (storeArena, levelArena); codes is the build's own.
    DeviceBuffer positions, shape, sh, codes, starts;
    DeviceBuffer mPositions, mShape, mSh, cells;
    DeviceBuffer storeArena, levelArena;
    ~lrt_lod() {
        DeviceScope scope(device);
        for (DeviceBuffer* b : {&codes, &storeArena, &levelArena}) release(*b);
    }
};

// One instance's drawn cloud and its cut's scratch: status words, then the
// drawn count, the merged count and the error word.
struct LodCutFrame {
    DeviceBuffer positions, shape, sh, status;
    uint32_t capacity = 0, shWords = 0;
    lrt_gpu_splats cloud{};
};

void release_cut_frames(lrt_rast* r) {
    for (LodCutFrame* f : r->cutFrames) {
        for (DeviceBuffer* b : {&f->positions, &f->shape, &f->sh, &f->status}) release(*b);
        delete f;
    }
    r->cutFrames.clear();
}

namespace {

uint32_t sh_words_for(uint32_t rest) { return (rest * 3 + 1) / 2; }

// One allocation for several buffers, each starting on a 256-byte boundary;
// the parts point into `arena` and are not freed on their own.
cudaError_t carve(DeviceBuffer& arena, std::initializer_list<std::pair<DeviceBuffer*, size_t>> parts) {
    size_t total = 0;
    for (const auto& p : parts) total += (std::max<size_t>(p.second, 16) + 255) & ~size_t{255};
    const cudaError_t e = ensure(arena, total);
    if (e != cudaSuccess) return e;
    size_t at = 0;
    for (const auto& p : parts) {
        p.first->ptr = static_cast<char*>(arena.ptr) + at;
        p.first->bytes = std::max<size_t>(p.second, 16);
        at += (p.first->bytes + 255) & ~size_t{255};
    }
    return cudaSuccess;
}

LodSplatArrays arrays_of(DeviceBuffer& positions, DeviceBuffer& shape, DeviceBuffer& sh) {
    return {static_cast<float4*>(positions.ptr), static_cast<uint4*>(shape.ptr), static_cast<uint32_t*>(sh.ptr)};
}

lrt_gpu_splats view_of(uint32_t count, uint32_t rest, uint32_t shWords, const void* positions, const void* shape,
                       const void* sh) {
    lrt_gpu_splats s{};
    s.count = count;
    s.rest_per_colour = rest;
    s.sh_words = shWords;
    s.positions = positions;
    s.shape = shape;
    s.sh = sh;
    return s;
}

// Scratch bytes of one cut: the cut's per-block bitmasks and counts, then 4
// words: the drawn count, the merged count and an always-zero error word.
size_t cut_status_bytes(uint32_t items) { return lrt::lod_cut_scratch_bytes(items) + 16; }

// The cut's parameters for one instance in this view (Lod.cpp:400-426): the
// eye in the cloud's space, and pixels per unit (the transform's largest
// column scale applies to orthographic sizes only).
LodCutParams cut_params(const lrt_lod& lod, const lrt_projection& pr, const lrt_lod_instance& inst, float threshold,
                        uint32_t capacity) {
    LodCutParams c{};
    c.merged = lod.merged;
    c.count = lod.count;
    c.levels = lod.levels;
    c.coarsest = lod.coarsest;
    for (uint32_t l = 0; l <= lod.levels; ++l) c.levelBase[l] = lod.levelBase[l];
    c.shWords = lod.shWords;
    c.capacity = capacity;
    c.ortho = pr.orthographic != 0 ? 1u : 0u;
    for (int k = 0; k < 3; ++k) c.lo[k] = lod.boundsLo[k];
    c.extent = lod.extent;
    double eye[3];
    eye_in_object(inst.object_to_world, pr.eye_world, eye);
    for (int k = 0; k < 3; ++k) c.eye[k] = static_cast<float>(eye[k]);
    const double* m = inst.object_to_world;
    double scale = 0.0;
    for (int col = 0; col < 3; ++col)
        scale = std::max(scale, std::sqrt(m[col] * m[col] + m[4 + col] * m[4 + col] + m[8 + col] * m[8 + col]));
    c.pixelsPerUnit = static_cast<float>(pr.orthographic != 0 ? pr.focal_x * scale : pr.focal_x);
    c.threshold = inst.threshold >= 0.0f ? inst.threshold : threshold;
    return c;
}

int run_cut(lrt_rast* r, const lrt_lod& lod, LodCutFrame& frame, const LodCutParams& c, uint32_t* hostCounts,
            cudaStream_t stream) {
    const uint32_t items = lod.merged + lod.count;
    const size_t statusBytes = cut_status_bytes(items);
    LRT_CUDA(r, ensure(frame.status, statusBytes), "cut scratch");
    uint32_t* counts = reinterpret_cast<uint32_t*>(static_cast<char*>(frame.status.ptr) + statusBytes - 16);
    LRT_CUDA(r, cudaMemsetAsync(counts, 0, 16, stream), "cut scratch");
    LodSplatArrays merged = {static_cast<float4*>(lod.mPositions.ptr), static_cast<uint4*>(lod.mShape.ptr),
                             static_cast<uint32_t*>(lod.mSh.ptr)};
    LodSplatArrays store = {static_cast<float4*>(lod.positions.ptr), static_cast<uint4*>(lod.shape.ptr),
                            static_cast<uint32_t*>(lod.sh.ptr)};
    LRT_CUDA(r, lrt::launch_lod_cut(c, static_cast<const uint32_t*>(lod.cells.ptr),
                                    static_cast<const uint32_t*>(lod.codes.ptr), merged, store,
                                    arrays_of(frame.positions, frame.shape, frame.sh), frame.status.ptr, counts,
                                    stream),
             "cut");
    LRT_CUDA(r, cudaMemcpyAsync(hostCounts, counts, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream), "cut counts");
    return LRT_OK;
}

int size_frame(lrt_rast* r, LodCutFrame& frame, uint32_t capacity, uint32_t shWords) {
    if (frame.capacity >= capacity && frame.shWords == shWords && frame.positions.ptr != nullptr) return LRT_OK;
    capacity = std::max(capacity, 1u);
    LRT_CUDA(r, ensure(frame.positions, size_t{capacity} * 16), "cut cloud");
    LRT_CUDA(r, ensure(frame.shape, size_t{capacity} * 16), "cut cloud");
    LRT_CUDA(r, ensure(frame.sh, size_t{capacity} * shWords * 4), "cut cloud");
    frame.capacity = capacity;
    frame.shWords = shWords;
    return LRT_OK;
}

}  // namespace

extern "C" {

int lrt_lod_build_settings_default(lrt_lod_build_settings* out) {
    if (out == nullptr) return LRT_INVALID_ARGUMENT;
    out->max_group_fraction = 0.5f;
    out->coarsest_level = 1;
    out->chunk_splats = 1u << 16;
    out->reserved = 0;
    return LRT_OK;
}

int lrt_lod_build(lrt_rast* r, const lrt_gpu_splats* cloud, const float* bounds,
                  const lrt_lod_build_settings* settingsIn, lrt_lod** out, void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (out == nullptr || cloud == nullptr) return fail(r, LRT_INVALID_ARGUMENT, "null cloud or result");
    *out = nullptr;
    const uint32_t n = cloud->count;
    if (n == 0) return fail(r, LRT_INVALID_ARGUMENT, "an empty cloud has no levels of detail");
    const uint32_t rest = cloud->rest_per_colour;
    if (rest != 0 && rest != 3 && rest != 8 && rest != 15)
        return fail(r, LRT_INVALID_ARGUMENT, "rest_per_colour must be 0, 3, 8 or 15");
    if (cloud->sh_words < sh_words_for(rest)) return fail(r, LRT_INVALID_ARGUMENT, "sh_words too small for rest_per_colour");
    if (cloud->positions == nullptr || cloud->shape == nullptr || (cloud->sh_words > 0 && cloud->sh == nullptr))
        return fail(r, LRT_INVALID_ARGUMENT, "null cloud buffers");
    if (n > (1u << 30)) return fail(r, LRT_INVALID_ARGUMENT, "too many splats");
    lrt_lod_build_settings settings;
    lrt_lod_build_settings_default(&settings);
    if (settingsIn != nullptr) settings = *settingsIn;
    const uint32_t coarsest = std::clamp<uint32_t>(settings.coarsest_level, 1, kLodLevels);
    const uint32_t shWords = cloud->sh_words;

    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    std::unique_ptr<lrt_lod> lod(new lrt_lod());
    lod->device = r->device;
    lod->count = n;
    lod->restPerColour = rest;
    lod->shWords = shWords;
    lod->coarsest = coarsest;
    lod->chunkSplats = std::max<uint32_t>(settings.chunk_splats, 1u);
    LodBuildScratch& t = r->lodBuild;   // kept between builds: a build allocates only what it returns
    LRT_CUDA(r, ensure(t.globals, sizeof(LodGlobals)), "lod buffers");
    LRT_CUDA(r, ensure(t.partial, std::max<size_t>(lrt::lod_bounds_partial_bytes(), 64)), "lod buffers");
    for (DeviceBuffer* b : {&t.keys, &t.keysAlt, &t.order, &t.orderAlt}) LRT_CUDA(r, ensure(*b, size_t{n} * 4), "lod buffers");
    LRT_CUDA(r, ensure(t.sortScratch, lrt::sort_scratch_bytes(n, 30)), "lod buffers");
    LRT_CUDA(r, ensure(t.err, 16), "lod buffers");
    LRT_CUDA(r,
             carve(lod->storeArena,
                   {{&lod->positions, size_t{n} * 16}, {&lod->shape, size_t{n} * 16}, {&lod->sh, size_t{n} * shWords * 4}}),
             "lod buffers");

    LodGlobals* globals = static_cast<LodGlobals*>(t.globals.ptr);
    uint32_t* err = static_cast<uint32_t*>(t.err.ptr);
    LodGlobals init{};
    init.count = n;
    LRT_CUDA(r, cudaMemcpyAsync(globals, &init, sizeof(init), cudaMemcpyHostToDevice, stream), "lod upload");
    LRT_CUDA(r, cudaMemsetAsync(err, 0, 16, stream), "lod upload");
    const float* given = nullptr;
    if (bounds != nullptr) {
        LRT_CUDA(r, cudaMemcpyAsync(t.partial.ptr, bounds, 6 * sizeof(float), cudaMemcpyHostToDevice, stream),
                 "lod upload");
        given = static_cast<const float*>(t.partial.ptr);
    }
    const float4* srcPositions = static_cast<const float4*>(cloud->positions);
    LRT_CUDA(r, lrt::launch_lod_bounds(srcPositions, n, given, globals, static_cast<float*>(t.partial.ptr), stream),
             "lod bounds");
    LRT_CUDA(r, lrt::launch_lod_morton(srcPositions, n, globals, static_cast<uint32_t*>(t.keys.ptr),
                                       static_cast<uint32_t*>(t.order.ptr), stream),
             "lod morton");
    bool inAlt = false;
    LRT_CUDA(r, lrt::launch_sort_u32(static_cast<uint32_t*>(t.keys.ptr), static_cast<uint32_t*>(t.keysAlt.ptr),
                                     static_cast<uint32_t*>(t.order.ptr), static_cast<uint32_t*>(t.orderAlt.ptr),
                                     &globals->count, n, 0, 30, t.sortScratch.ptr, err, &inAlt, stream),
             "lod sort");
    // The sorted codes stay with the cloud.
    std::swap(lod->codes, inAlt ? t.keysAlt : t.keys);
    const uint32_t* codes = static_cast<const uint32_t*>(lod->codes.ptr);
    const uint32_t* order = static_cast<const uint32_t*>((inAlt ? t.orderAlt : t.order).ptr);
    LodSplatArrays store = arrays_of(lod->positions, lod->shape, lod->sh);
    LRT_CUDA(r, lrt::launch_lod_reorder(order, codes, n, shWords, srcPositions, static_cast<const uint4*>(cloud->shape),
                                        static_cast<const uint32_t*>(cloud->sh), store, globals, stream),
             "lod reorder");
    LodGlobals host{};
    uint32_t hostErr = 0;
    LRT_CUDA(r, cudaMemcpyAsync(&host, globals, sizeof(host), cudaMemcpyDeviceToHost, stream), "lod counts");
    LRT_CUDA(r, cudaMemcpyAsync(&hostErr, err, sizeof(hostErr), cudaMemcpyDeviceToHost, stream), "lod counts");
    LRT_CUDA(r, cudaStreamSynchronize(stream), "lod counts");
    if (hostErr != 0) return fail(r, LRT_DEVICE_FAILURE, "lod sort: a look-back wait ran out");

    // Every level's group count; the finest level worth storing (Lod.cpp:200-211).
    uint32_t groups[kLodLevels + 1] = {};
    uint64_t running = 1;
    for (uint32_t level = 1; level <= kLodLevels; ++level) {
        running += host.firstLevel[level];
        groups[level] = static_cast<uint32_t>(running);
    }
    uint32_t finest = coarsest;
    for (uint32_t level = coarsest; level <= kLodLevels; ++level) {
        if (static_cast<float>(groups[level]) > settings.max_group_fraction * static_cast<float>(n) &&
            level > coarsest)
            break;
        finest = level;
    }
    const uint32_t levels = finest - coarsest + 1;
    lod->finest = finest;
    lod->levels = levels;
    lod->levelBase[0] = 0;
    for (uint32_t l = 0; l < levels; ++l) lod->levelBase[l + 1] = lod->levelBase[l] + groups[coarsest + l];
    const uint32_t merged = lod->levelBase[levels];
    lod->merged = merged;
    for (int k = 0; k < 3; ++k) lod->boundsLo[k] = host.lo[k], lod->boundsHi[k] = host.hi[k];
    lod->extent = host.extent;
    const uint32_t stride = kLodMomentsHead + 3 * rest;
    const uint32_t finestGroups = groups[finest];
    LRT_CUDA(r,
             carve(lod->levelArena, {{&lod->mPositions, size_t{merged} * 16}, {&lod->mShape, size_t{merged} * 16},
                                     {&lod->mSh, size_t{merged} * shWords * 4}, {&lod->cells, size_t{merged} * 4},
                                     {&lod->starts, size_t{finestGroups} * 4}}),
             "lod levels");
    LRT_CUDA(r, ensure(t.firstChild, size_t{merged} * 4), "lod levels");
    LRT_CUDA(r, ensure(t.moments, size_t{merged} * stride * 4), "lod levels");
    // One status region per compaction: the finest level's over the splats,
    // each coarser level's over the groups of the level below it.
    const uint32_t threads = lrt::lod_compaction_threads();
    std::vector<size_t> statusAt(levels + 1, 0);
    statusAt[levels - 1] = 0;
    size_t statusBytes = lrt::compaction_status_bytes(n, threads);
    for (uint32_t l = levels - 1; l-- > 0;) {
        statusAt[l] = statusBytes;
        statusBytes += lrt::compaction_status_bytes(groups[coarsest + l + 1], threads);
    }
    LRT_CUDA(r, ensure(t.status, statusBytes), "lod levels");
    LRT_CUDA(r, cudaMemsetAsync(t.status.ptr, 0, statusBytes, stream), "lod levels");
    char* status = static_cast<char*>(t.status.ptr);
    uint32_t* cells = static_cast<uint32_t*>(lod->cells.ptr);
    uint32_t* firstChild = static_cast<uint32_t*>(t.firstChild.ptr);
    float* moments = static_cast<float*>(t.moments.ptr);
    LRT_CUDA(r, lrt::launch_lod_finest_groups(codes, n, finest, finestGroups, static_cast<uint32_t*>(lod->starts.ptr),
                                              cells + lod->levelBase[levels - 1], status + statusAt[levels - 1],
                                              &globals->groupTotals[finest], err, stream),
             "lod groups");
    for (uint32_t l = levels - 1; l-- > 0;) {
        const uint32_t level = coarsest + l;
        LRT_CUDA(r, lrt::launch_lod_parent_groups(cells + lod->levelBase[l + 1], groups[level + 1], groups[level],
                                                  cells + lod->levelBase[l], firstChild + lod->levelBase[l],
                                                  status + statusAt[l], &globals->groupTotals[level], err, stream),
                 "lod groups");
    }
    // Moments from the finest stored level up (Lod.cpp:213-266), then one
    // Gaussian per group of every level.
    LRT_CUDA(r, lrt::launch_lod_leaf_moments(store, n, rest, shWords, static_cast<const uint32_t*>(lod->starts.ptr),
                                             finestGroups, moments + size_t{lod->levelBase[levels - 1]} * stride,
                                             stream),
             "lod moments");
    for (uint32_t l = levels - 1; l-- > 0;) {
        const uint32_t level = coarsest + l;
        LRT_CUDA(r, lrt::launch_lod_merge_moments(firstChild + lod->levelBase[l], groups[level], groups[level + 1],
                                                  moments + size_t{lod->levelBase[l + 1]} * stride,
                                                  moments + size_t{lod->levelBase[l]} * stride, stride, stream),
                 "lod moments");
    }
    LRT_CUDA(r, lrt::launch_lod_finalize(moments, merged, rest, shWords,
                                         arrays_of(lod->mPositions, lod->mShape, lod->mSh), stream),
             "lod finalize");
    LodGlobals after{};
    LRT_CUDA(r, cudaMemcpyAsync(&after, globals, sizeof(after), cudaMemcpyDeviceToHost, stream), "lod check");
    LRT_CUDA(r, cudaMemcpyAsync(&hostErr, err, sizeof(hostErr), cudaMemcpyDeviceToHost, stream), "lod check");
    LRT_CUDA(r, cudaStreamSynchronize(stream), "lod check");
    if (hostErr != 0) return fail(r, LRT_DEVICE_FAILURE, "lod groups: a look-back wait ran out");
    for (uint32_t level = coarsest; level <= finest; ++level)
        if (after.groupTotals[level] != groups[level])
            return fail(r, LRT_DEVICE_FAILURE, "lod groups: a level's compaction disagrees with its count");
    *out = lod.release();
    return LRT_OK;
}

void lrt_lod_destroy(lrt_lod* lod) { delete lod; }

int lrt_lod_get_info(const lrt_lod* lod, lrt_lod_info* out) {
    if (lod == nullptr || out == nullptr) return LRT_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    out->count = lod->count;
    out->rest_per_colour = lod->restPerColour;
    out->sh_words = lod->shWords;
    out->levels = lod->levels;
    out->coarsest = lod->coarsest;
    out->finest = lod->finest;
    out->merged = lod->merged;
    out->chunk_splats = lod->chunkSplats;
    for (int k = 0; k < 3; ++k) out->bounds_lo[k] = lod->boundsLo[k], out->bounds_hi[k] = lod->boundsHi[k];
    out->extent = lod->extent;
    for (uint32_t l = 0; l < lod->levels; ++l) out->level_groups[l] = lod->levelBase[l + 1] - lod->levelBase[l];
    return LRT_OK;
}

int lrt_lod_splats(const lrt_lod* lod, lrt_gpu_splats* out, const uint32_t** codes) {
    if (lod == nullptr || out == nullptr) return LRT_INVALID_ARGUMENT;
    *out = view_of(lod->count, lod->restPerColour, lod->shWords, lod->positions.ptr, lod->shape.ptr, lod->sh.ptr);
    if (codes != nullptr) *codes = static_cast<const uint32_t*>(lod->codes.ptr);
    return LRT_OK;
}

int lrt_lod_level(const lrt_lod* lod, uint32_t index, uint32_t* level, lrt_gpu_splats* gaussians,
                  const uint32_t** cells) {
    if (lod == nullptr || index >= lod->levels) return LRT_INVALID_ARGUMENT;
    const uint32_t first = lod->levelBase[index];
    const uint32_t n = lod->levelBase[index + 1] - first;
    if (level != nullptr) *level = lod->coarsest + index;
    if (gaussians != nullptr)
        *gaussians = view_of(n, lod->restPerColour, lod->shWords, static_cast<const char*>(lod->mPositions.ptr) + size_t{first} * 16,
                             static_cast<const char*>(lod->mShape.ptr) + size_t{first} * 16,
                             static_cast<const char*>(lod->mSh.ptr) + size_t{first} * lod->shWords * 4);
    if (cells != nullptr) *cells = static_cast<const uint32_t*>(lod->cells.ptr) + first;
    return LRT_OK;
}

int lrt_lod_starts(const lrt_lod* lod, const uint32_t** starts, uint32_t* groups) {
    if (lod == nullptr) return LRT_INVALID_ARGUMENT;
    if (starts != nullptr) *starts = static_cast<const uint32_t*>(lod->starts.ptr);
    if (groups != nullptr) *groups = lod->levelBase[lod->levels] - lod->levelBase[lod->levels - 1];
    return LRT_OK;
}

int lrt_lod_select(lrt_rast* r, const lrt_projection* pr, const lrt_lod_instance* instances, uint32_t count,
                   float threshold, lrt_splat_instance* out, uint32_t* outCount, lrt_cut_stats* stats,
                   void* streamPtr) {
    if (r == nullptr) return LRT_INVALID_ARGUMENT;
    r->error.clear();
    if (pr == nullptr || outCount == nullptr || (count > 0 && (instances == nullptr || out == nullptr)))
        return fail(r, LRT_INVALID_ARGUMENT, "null projection, instances or result");
    *outCount = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const lrt_lod* lod = instances[k].cloud;
        if (lod != nullptr && lod->count > 0 && lod->device != r->device)
            return fail(r, LRT_INVALID_ARGUMENT, "a cloud lives on another device");
    }
    DeviceScope scope(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    // An enqueued frame may still be drawing the clouds this call rewrites.
    if (r->frameDoneSet) LRT_CUDA(r, cudaStreamWaitEvent(stream, r->frameDone, 0), "frame order");
    while (r->cutFrames.size() < count) r->cutFrames.push_back(new LodCutFrame());
    LRT_CUDA(r, ensure_host(r, size_t{count} * 4 * sizeof(uint32_t) + 16), "cut counts");
    uint32_t* host = static_cast<uint32_t*>(r->metricHost);
    std::vector<LodCutParams> params(count);
    std::vector<uint8_t> active(count, 0);
    for (uint32_t k = 0; k < count; ++k) {
        const lrt_lod* lod = instances[k].cloud;
        if (lod == nullptr || lod->count == 0) continue;
        LodCutFrame& frame = *r->cutFrames[k];
        // Drawn items never outnumber the splats: each place is drawn once,
        // and a merged Gaussian stands for at least one splat.
        if (int e = size_frame(r, frame, std::max(frame.capacity, lod->count), lod->shWords); e != LRT_OK) return e;
        params[k] = cut_params(*lod, *pr, instances[k], threshold, frame.capacity);
        active[k] = 1;
        if (int e = run_cut(r, *lod, frame, params[k], host + 4 * k, stream); e != LRT_OK) return e;
    }
    LRT_CUDA(r, cudaStreamSynchronize(stream), "cut counts");
    bool again = false;
    for (uint32_t k = 0; k < count; ++k) {
        if (!active[k]) continue;
        if (host[4 * k + 2] != 0) return fail(r, LRT_DEVICE_FAILURE, "cut: a look-back wait ran out");
        if (host[4 * k] > params[k].capacity) {
            LodCutFrame& frame = *r->cutFrames[k];
            if (int e = size_frame(r, frame, host[4 * k], instances[k].cloud->shWords); e != LRT_OK) return e;
            params[k].capacity = frame.capacity;
            if (int e = run_cut(r, *instances[k].cloud, frame, params[k], host + 4 * k, stream); e != LRT_OK) return e;
            again = true;
        }
    }
    if (again) LRT_CUDA(r, cudaStreamSynchronize(stream), "cut counts");
    uint32_t written = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const lrt_lod* lod = instances[k].cloud;
        lrt_cut_stats s{};
        if (active[k]) {
            const uint32_t drawn = host[4 * k], mergedDrawn = host[4 * k + 1];
            if (host[4 * k + 2] != 0 || drawn > params[k].capacity)
                return fail(r, LRT_DEVICE_FAILURE, "cut: the drawn count passed its cloud");
            s.splats = drawn - mergedDrawn;
            s.merged = mergedDrawn;
            s.available = lod->count;
            LodCutFrame& frame = *r->cutFrames[k];
            frame.cloud = view_of(drawn, lod->restPerColour, lod->shWords, frame.positions.ptr, frame.shape.ptr,
                                  frame.sh.ptr);
            if (drawn > 0) {
                lrt_splat_instance& o = out[written++];
                o.splats = &frame.cloud;
                std::memcpy(o.object_to_world, instances[k].object_to_world, sizeof(o.object_to_world));
                o.edit = instances[k].edit;
            }
        }
        if (stats != nullptr) stats[k] = s;
    }
    *outCount = written;
    return LRT_OK;
}

}  // extern "C"
