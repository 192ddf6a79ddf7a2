// The rasteriser handle's state and the small host helpers its entry points
// share (raster.cu, lod_host.cu). Private to the library.
#pragma once

#include "../../include/lrt_raster.h"
#include "kernels.cuh"
#include "raster_common.cuh"

#include <cmath>
#include <memory>
#include <string>
#include <algorithm>
#include <vector>

struct LodCutFrame;   // lod_host.cu: one instance's cut cloud

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
};

// A level-of-detail build's temporaries (lod_host.cu): the bounds and
// counters, the Morton sort's keys, indices and scratch, the look-back
// status words, each group's first child and moments, the error word.
struct LodBuildScratch {
    DeviceBuffer globals, partial, keys, keysAlt, order, orderAlt, sortScratch, status, firstChild, moments, err;
};

struct lrt_rast {
    int device = 0;
    std::string error;
    DeviceBuffer proj, rects, touched, keys;            // per slot
    DeviceBuffer pairs, pairsAlt;                        // per pair
    DeviceBuffer ranges;                                 // per tile
    DeviceBuffer tileOrder;                              // per tile: the blend's launch order
    DeviceBuffer scanScratch, sortScratch;               // look-back status words, tickets
    DeviceBuffer counters;                               // visible, pairs, err, algo err
    DeviceBuffer algoKeysAlt, algoValsAlt;               // lrt_radix_sort's ping-pong buffers
    DeviceBuffer depthWords, depthWordsAlt, splatAux;    // per slot: depth words (two-step frames), aux words
    DeviceBuffer rowTable;                               // large splats' rows (first column, count)
    uint32_t rowCap = 0;                                 // its entries
    lrt::SortFault sortFault;                            // lrt_radix_sort's planted fault (tests only)
    DeviceBuffer filterCameras, filterScratch;           // lrt_rast_filter3d's cameras and lowest rate
    uint32_t* hostCounters = nullptr;                    // pinned
    uint32_t* hostCountersDev = nullptr;                 // the device's address of hostCounters
    // ev[0..5]: a frame's stage times; ev[6]: an enqueued training frame's
    // counts copied to the host; ev[7..9]: the training backward's times.
    cudaEvent_t ev[10] = {};
    uint32_t splatCap = 0, pairCap = 0, tileCap = 0;
    lrt_debug_view debug{};
    // Training: what the backward pass needs from its forward.
    DeviceBuffer pairValues, pairValuesAlt, pairOffsets, pixState, pixLast, partials;
    DeviceBuffer metricScratch;                          // parity metrics: histograms, row errors
    DeviceBuffer lossScratch;                            // the L1 loss's per-block sums
    // Training batches (train_batch.cu): colour gradients, every view's view
    // and frame parameters with the chunks' queues, losses with no caller
    // buffer; their pair capacity.
    DeviceBuffer trainBatchGrad, trainBatchViews, trainBatchLoss;
    uint32_t trainBatchPairCap = 0;
    void* metricHost = nullptr;                          // pinned readback of the metrics
    size_t metricHostBytes = 0;
    bool trainReady = false;
    bool trainPending = false;   // the forward's counts and status are not read yet
    cudaStream_t pendingStream = nullptr;
    bool trainSized = false;     // a training frame has run with a wait
    uint32_t trainSlots = 0, trainWidth = 0, trainHeight = 0;   // that frame's shape
    uint32_t trainSeenPairs = 0;  // the pairs of the last training frame whose counts were read
    lrt_train_params trainParams{};
    lrt::FrameParams trainFrame{};
    lrt::BlendParams trainBlend{};
    const uint64_t* trainSorted = nullptr;
    const uint32_t* trainSortedValues = nullptr;   // emit index per sorted pair (value layout)
    const uint32_t* trainEmitSlot = nullptr;       // slot per emit index (low-field layout)
    uint32_t trainPairs = 0;
    bool backwardTimed = false;   // ev[7..9] hold a training backward's times
    // Plain frames enqueued by lrt_rast_render_async: their counts land in a
    // ring of pinned slots, each with the event that marks its frame done.
    static constexpr uint32_t kRing = 16;
    uint32_t* ringHost = nullptr;               // pinned, 4 words per slot
    uint32_t* ringHostDev = nullptr;            // the device's address of ringHost
    cudaEvent_t ringEvent[kRing] = {};
    uint32_t ringCap[kRing] = {};               // the pair capacity each frame ran with
    uint64_t ringHead = 0, ringTail = 0;        // next slot to fill; oldest slot not read
    bool plainSized = false;                    // a plain frame of this shape has run with a wait
    uint32_t plainSlots = 0, plainWidth = 0, plainHeight = 0, plainSeenPairs = 0;
    uint32_t asyncOverflows = 0, asyncTimeouts = 0;   // among the frames read since the last settle
    uint32_t asyncVisible = 0, asyncPairs = 0, asyncSplats = 0;   // the last frame read
    cudaEvent_t frameDone = nullptr;            // end of the last frame, on its stream
    bool frameDoneSet = false;
    // Batches of views.
    struct Batch {
        cudaStream_t stream = nullptr;
        cudaEvent_t in = nullptr, out = nullptr, start = nullptr, end = nullptr;
        DeviceBuffer records, ranges, params, counters, queue;
        void* hostParams = nullptr;   // pinned: FrameParams per (view, instance), then ViewParams per view
        size_t hostParamsBytes = 0;
        uint32_t* hostCounters = nullptr;   // pinned: 4 words per chunk
        uint32_t hostCounterChunks = 0;
        uint64_t generation = 0;            // bumped whenever a buffer the graph uses moves
        cudaGraphExec_t graph = nullptr;
        uint64_t graphKey = 0, graphGeneration = 0;
        bool graphFailed = false;
        std::vector<std::pair<uint64_t, std::pair<uint32_t, uint32_t>>> tuned;   // shape -> (views per chunk, blocks/SM)
    } batch;
    // Training batches (train_batch.cu): a stream of their own, the views'
    // and frames' parameters staged in pinned memory, per-chunk counters read
    // back once a step, the captured step and the tuned shapes.
    struct TrainBatch {
        cudaStream_t stream = nullptr;
        cudaEvent_t in = nullptr, out = nullptr, start = nullptr, end = nullptr;
        DeviceBuffer counters;
        void* hostParams = nullptr;        // pinned: ViewParams then FrameParams for every view
        size_t hostParamsBytes = 0;
        uint32_t* hostCounters = nullptr;  // pinned: 4 words per chunk
        uint32_t hostCounterChunks = 0;
        uint64_t generation = 0;           // bumped whenever a buffer the graph uses moves
        cudaGraphExec_t graph = nullptr;
        uint64_t graphKey = 0, graphGeneration = 0;
        bool graphFailed = false;
        std::vector<std::pair<uint64_t, std::pair<uint32_t, uint32_t>>> tuned;   // shape -> (views per chunk, blocks/SM)
        uint32_t fixedChunk = 0, fixedBlocks = 0;   // set by the test hook: no tuning
    } trainBatch;
    // Levels of detail: the clouds the last lrt_lod_select made, one per
    // instance, rewritten by the next call, and the builds' temporaries, kept
    // from one build to the next (lod_host.cu).
    std::vector<LodCutFrame*> cutFrames;
    LodBuildScratch lodBuild;
};

// lod_host.cu: frees the cut clouds (called by lrt_rast_destroy).
void release_cut_frames(lrt_rast* r);

namespace {

using lrt::BlendParams;
using lrt::FrameParams;
using lrt::ProjRecord;

inline int fail(lrt_rast* r, int code, const std::string& message) {
    if (r != nullptr) r->error = message;
    return code;
}

inline int cuda_fail(lrt_rast* r, cudaError_t e, const char* what) {
    const int code = e == cudaErrorMemoryAllocation ? LRT_OUT_OF_MEMORY : LRT_DEVICE_FAILURE;
    return fail(r, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define LRT_CUDA(r, call, what)                         \
    do {                                                \
        const cudaError_t e_ = (call);                  \
        if (e_ != cudaSuccess) return cuda_fail(r, e_, what); \
    } while (0)

// TileRasterizer.cpp:26-32
inline uint32_t grow(uint32_t have, uint32_t need) {
    uint64_t size = std::max<uint32_t>(have, 1024);
    while (size < need) size = size * 3 / 2;
    return static_cast<uint32_t>(std::min<uint64_t>(size, 0xFFFFFFFFull));
}

inline cudaError_t ensure(DeviceBuffer& b, size_t bytes) {
    if (b.bytes >= bytes && b.ptr != nullptr) return cudaSuccess;
    // Work still queued (an enqueued frame, a backward that returned without
    // waiting) may read the old buffer: it finishes before the buffer goes.
    if (b.ptr != nullptr) {
        cudaDeviceSynchronize();
        cudaFree(b.ptr);
    }
    b.ptr = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.ptr, std::max<size_t>(bytes, 16));
    if (e == cudaSuccess) b.bytes = std::max<size_t>(bytes, 16);
    return e;
}

// Where a batch's ViewParams start in its parameter block: after the
// FrameParams of every (view, instance), rounded up to 16 bytes, since a
// ViewParams holds 8-byte pointers (a FrameParams is 212 bytes).
inline size_t view_params_offset(uint32_t launches) {
    return (size_t{launches} * sizeof(lrt::FrameParams) + 15) & ~size_t{15};
}

inline cudaError_t ensure_host(lrt_rast* r, size_t bytes) {
    if (r->metricHostBytes >= bytes && r->metricHost != nullptr) return cudaSuccess;
    if (r->metricHost != nullptr) cudaFreeHost(r->metricHost);
    r->metricHost = nullptr;
    r->metricHostBytes = 0;
    cudaError_t e = cudaMallocHost(&r->metricHost, bytes);
    if (e == cudaSuccess) r->metricHostBytes = bytes;
    return e;
}

inline void release(DeviceBuffer& b) {
    if (b.ptr != nullptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
}

// FrameParams.h:18-24
inline uint32_t bits_for(uint64_t values) {
    uint32_t bits = 1;
    while (bits < 32 && (uint64_t{1} << bits) < values) ++bits;
    return bits;
}

struct M4 {
    double m[16];
    double at(int r, int c) const { return m[r * 4 + c]; }
};

inline M4 mul4(const double* a, const double* b) {
    M4 o{};
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += a[r * 4 + k] * b[k * 4 + c];
            o.m[r * 4 + c] = s;
        }
    return o;
}

// The eye in the instance's own space: inverse(objectToWorld) applied to the
// world eye (TileRasterizer.cpp:298-299, aofx::xform::inverseAffine).
inline void eye_in_object(const double* m, const double* eye, double out[3]) {
    auto at = [&](int r, int c) { return m[r * 4 + c]; };
    const double a00 = at(0, 0), a01 = at(0, 1), a02 = at(0, 2);
    const double a10 = at(1, 0), a11 = at(1, 1), a12 = at(1, 2);
    const double a20 = at(2, 0), a21 = at(2, 1), a22 = at(2, 2);
    const double c00 = a11 * a22 - a12 * a21;
    const double c01 = a12 * a20 - a10 * a22;
    const double c02 = a10 * a21 - a11 * a20;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    const double inv = std::fabs(det) > 1e-18 ? 1.0 / det : 0.0;
    const double i00 = c00 * inv, i01 = (a02 * a21 - a01 * a22) * inv, i02 = (a01 * a12 - a02 * a11) * inv;
    const double i10 = c01 * inv, i11 = (a00 * a22 - a02 * a20) * inv, i12 = (a02 * a10 - a00 * a12) * inv;
    const double i20 = c02 * inv, i21 = (a01 * a20 - a00 * a21) * inv, i22 = (a00 * a11 - a01 * a10) * inv;
    const double tx = at(0, 3), ty = at(1, 3), tz = at(2, 3);
    const double b0 = -(i00 * tx + i01 * ty + i02 * tz);
    const double b1 = -(i10 * tx + i11 * ty + i12 * tz);
    const double b2 = -(i20 * tx + i21 * ty + i22 * tz);
    out[0] = i00 * eye[0] + i01 * eye[1] + i02 * eye[2] + b0;
    out[1] = i10 * eye[0] + i11 * eye[1] + i12 * eye[2] + b1;
    out[2] = i20 * eye[0] + i21 * eye[1] + i22 * eye[2] + b2;
}

inline float event_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) return 0.0f;
    return ms;
}

struct DeviceScope {
    int previous = -1;
    explicit DeviceScope(int device) {
        if (cudaGetDevice(&previous) == cudaSuccess && previous != device) {
            cudaSetDevice(device);
        } else {
            previous = -1;
        }
    }
    ~DeviceScope() {
        if (previous >= 0) cudaSetDevice(previous);
    }
};

// One cloud of a frame, whichever its kind, and the projection uniforms of a
// view of it (FrameParams.h:32-93).
struct CloudDesc {
    const lrt_gpu_splats* packed = nullptr;
    const lrt_train_params* train = nullptr;
    const lrt_point_instance* point = nullptr;   // points drawn as discs
    const double* objectToWorld = nullptr;
    const lrt_splat_edit* edit = nullptr;
    uint32_t count = 0;
};

inline constexpr double kIdentity[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};

inline FrameParams frame_params(const lrt_projection* pr, const lrt_render_settings* s, const CloudDesc& c, uint32_t tilesX,
                         uint32_t tilesY, uint32_t base) {
    FrameParams f{};
    f.width = s->width;
    f.height = s->height;
    f.tilesX = tilesX;
    f.tilesY = tilesY;
    f.focalX = static_cast<float>(pr->focal_x);
    f.focalY = static_cast<float>(pr->focal_y);
    f.centreX = static_cast<float>(pr->centre_x);
    f.centreY = static_cast<float>(pr->centre_y);
    f.nearZ = static_cast<float>(pr->near_z);
    f.farZ = static_cast<float>(pr->far_z);
    f.ortho = pr->orthographic ? 1u : 0u;
    f.antialias = s->antialias ? 1u : 0u;
    const M4 ov = mul4(pr->world_to_view, c.objectToWorld);
    for (int row = 0; row < 3; ++row)
        for (int col = 0; col < 4; ++col) f.m[row * 4 + col] = static_cast<float>(ov.at(row, col));
    double eye[3];
    eye_in_object(c.objectToWorld, pr->eye_world, eye);
    for (int a = 0; a < 3; ++a) f.eye[a] = static_cast<float>(eye[a]);
    f.count = c.count;
    f.base = base;
    if (c.train != nullptr) {
        f.restPerColour = 15;
        f.shWords = 24;
    } else if (c.packed != nullptr) {
        f.restPerColour = c.packed->rest_per_colour;
        f.shWords = c.packed->sh_words;
    }
    f.shLimit = s->max_sh_degree;
    f.writeDebug = 1;
    if (c.edit != nullptr) {
        const lrt_splat_edit& e = *c.edit;
        f.edit.active = e.active;
        f.edit.shape = e.shape;
        f.edit.mode = e.mode;
        f.edit.invert = e.invert;
        for (int a = 0; a < 3; ++a) {
            f.edit.centre[a] = e.centre[a];
            f.edit.size[a] = e.size[a];
            f.edit.tint[a] = e.tint[a];
        }
        f.edit.saturation = e.saturation;
        f.edit.brightness = e.brightness;
        f.edit.opacity = e.opacity;
        f.edit.minOpacity = e.min_opacity;
        f.edit.maxScale = e.max_scale;
    }
    return f;
}

}  // namespace
