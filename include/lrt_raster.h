/*
 * lrt_raster.h -- C-ABI of the B200 splat tile rasteriser.
 *
 * Drop-in for lucabRTrender's splat raster path: packed Gaussian clouds in
 * (the scene::GpuSplats layout), premultiplied linear colour and view-z depth
 * out (bottom row first), and the per-stage timings `lrt bench --stages`
 * prints. Every signature is plain C: device pointers and sizes, no C++ or
 * torch types, so a C++, Python (ctypes) or any other FFI host can bind it.
 *
 * Reference interfaces replaced (paths inside the lucabRTrender tree):
 *   lrt_rast_create        modules/render/src/TileRasterizer.cpp:59-103
 *                          (TileRasterizer::create)
 *   lrt_rast_render        modules/render/src/TileRasterizer.cpp:188-484
 *                          (TileRasterizer::render(const Projection&, ...))
 *   lrt_projection_for     modules/render/src/Camera.cpp:23-48 (projectionFor)
 *   lrt_camera_looking_at  modules/render/src/Camera.cpp:9-13 (Camera::lookingAt)
 *   lrt_prefix_sum         modules/gpu/src/algo/PrefixSum.cpp:58-88 (PrefixSum::apply)
 *   lrt_radix_sort         modules/gpu/src/algo/RadixSort.cpp:80-157 (RadixSort::sort)
 *   lrt_pack_splats        modules/scene/src/GpuClouds.cpp:151-226 and
 *                          shaders/lrt/scene/splat_decode.slang:20-91 (CloudLoader::upload,
 *                          host-side; the packed bytes are what the raster reads)
 *
 * Conventions (the reference's, shaders/lrt/splat/frame.slang:22-27):
 * +z forward, x right, y up; screen origin bottom-left; pixel centres at +0.5;
 * 16x16 tiles. Errors are returned as an lrt_status (the reference's
 * lrt::ErrorCode, modules/core/include/lrt/core/Error.h:14-26, plus OVERFLOW and
 * TIMEOUT for device-side capacity and bounded-wait failures); nothing throws,
 * and lrt_rast_last_error() gives the message. One calling thread per handle;
 * every call is ordered on the caller's CUDA stream.
 */
#ifndef LRT_RASTER_H
#define LRT_RASTER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LRT_ABI_VERSION 1u
#define LRT_TILE 16u

typedef enum lrt_status {
    LRT_OK = 0,
    LRT_UNKNOWN = 1,
    LRT_NOT_FOUND = 2,
    LRT_INVALID_ARGUMENT = 3,
    LRT_UNSUPPORTED = 4,
    LRT_IO_FAILURE = 5,
    LRT_DEVICE_FAILURE = 6,
    LRT_OUT_OF_MEMORY = 8,
    LRT_INTERNAL_ERROR = 10,
    /* Not in the reference's ErrorCode: a device-side capacity check failed
     * (more pairs were emitted than the pair buffer holds). */
    LRT_OVERFLOW = 11,
    /* A bounded device-side wait (decoupled look-back, bulk-copy barrier)
     * gave up; the kernel returned instead of spinning. */
    LRT_TIMEOUT = 12
} lrt_status;

/* Projection (modules/render/include/lrt/render/Camera.h:56-82), the part
 * the rasteriser reads. Row-major 4x4 acting on column vectors. */
typedef struct lrt_projection {
    double world_to_view[16];
    double focal_x, focal_y;     /* pixels per unit of x/z (perspective) or per unit (ortho) */
    double centre_x, centre_y;
    double near_z, far_z;
    double eye_world[3];
    uint32_t orthographic;
    uint32_t reserved;
} lrt_projection;

/* Lens + Camera (Camera.h:23-53). */
typedef struct lrt_lens {
    uint32_t orthographic;
    uint32_t reserved;
    double focal;              /* mm */
    double haperture;          /* mm */
    double vaperture;          /* mm */
    double near_z, far_z;
    double window_translate[2];
    double window_scale[2];
    double window_roll;        /* degrees, counter-clockwise */
} lrt_lens;

typedef struct lrt_camera {
    double camera_to_world[16];
    lrt_lens lens;
} lrt_camera;

/* SplatEdit (modules/render/include/lrt/render/TileRasterizer.h:29-50). */
typedef struct lrt_splat_edit {
    uint32_t active;
    uint32_t shape;   /* 0 box, 1 sphere */
    uint32_t mode;    /* 0 keep inside, 1 remove inside, 2 grade inside */
    uint32_t invert;
    float centre[3];
    float size[3];
    float tint[3];
    float saturation, brightness, opacity, min_opacity, max_scale;
} lrt_splat_edit;

/* scene::GpuSplats (modules/scene/include/lrt/scene/GpuClouds.h:41-76):
 *   positions  float4 per splat: xyz, linear opacity
 *   shape      uint32 x4 per splat: [0] smallest-three quaternion,
 *              [1] f16 log sx | f16 log sy << 16, [2] f16 log sz | f16 base r << 16,
 *              [3] f16 base g | f16 base b << 16
 *   sh         sh_words uint32 per splat: f16 rest coefficients, rgb per basis
 * All three are device pointers owned by the caller.
 *   filter3d   optional (null: off, the reference's behaviour): one float per
 *              splat, the variance of the Mip-Splatting 3D smoothing filter
 *              (Yu et al., "Mip-Splatting", CVPR 2024, section 4.1) in the
 *              cloud's own units, e.g. from lrt_rast_filter3d. When set, the
 *              projection widens each splat's scales to sqrt(s^2 + v) and
 *              scales its opacity by sqrt(prod s^2 / prod (s^2 + v)) before
 *              anything else reads them. No counterpart in the reference,
 *              which has only the 2D filter. */
typedef struct lrt_gpu_splats {
    uint32_t count;
    uint32_t rest_per_colour;   /* 0, 3, 8, 15 -> degree 0..3 */
    uint32_t sh_words;          /* (rest_per_colour * 3 + 1) / 2 */
    uint32_t reserved;
    const void* positions;
    const void* shape;
    const void* sh;
    const void* filter3d;
} lrt_gpu_splats;

/* SplatInstance (TileRasterizer.h:52-67) without the relight fields. */
typedef struct lrt_splat_instance {
    const lrt_gpu_splats* splats;
    double object_to_world[16];
    lrt_splat_edit edit;
} lrt_splat_instance;

/* scene::GpuPoints (GpuClouds.h:78-85): `count` points, positions float4
 * (x, y, z, 1) and colours two uint32 words each of fp16 halves, r | g << 16
 * and b | a << 16, linear. Device pointers. */
typedef struct lrt_gpu_points {
    uint32_t count;
    uint32_t reserved;
    const void* positions;
    const void* colours;
} lrt_gpu_points;

/* PointStyle (Points.h), the fields the disc route reads: size_mode 0 world
 * units, 1 pixels; size the diameter; constant_colour 1 draws every point
 * in colour[] (linear). The raster route's eye-dome lighting and surface
 * splatting need a rasterisation pipeline and are not part of this path. */
typedef struct lrt_point_style {
    uint32_t size_mode;
    float size;
    uint32_t constant_colour;
    float colour[3];
} lrt_point_style;

/* PointInstance (Points.h): points drawn as opaque discs, sorted with the
 * splats (shaders/lrt/splat/points_project.slang). */
typedef struct lrt_point_instance {
    const lrt_gpu_points* points;
    double object_to_world[16];
    lrt_point_style style;
} lrt_point_instance;

/* RenderSettings (TileRasterizer.h:105-118). */
typedef struct lrt_render_settings {
    uint32_t width, height;
    uint32_t antialias;
    uint32_t max_sh_degree;
    float background[4];        /* premultiplied, linear */
    uint32_t depth_mode;        /* 0 alpha-weighted mean, 1 first crossing of depth_threshold */
    float depth_threshold;
    uint32_t linearise;
    uint32_t time_stages;       /* record per-stage CUDA events into the stats */
} lrt_render_settings;

/* FrameStats (TileRasterizer.h:120-126). Stage times are CUDA-event times on
 * the render stream when time_stages is set; total_ms is host wall time.
 * Projection, the touched counts and pair emission are one kernel, reported
 * as project_ms (counts_ms and emit_ms are 0); the depth order is folded into
 * the pair sort's key, so that sort is reported under tile_sort_ms (with the
 * ranges) and depth_sort_ms is 0. */
typedef struct lrt_frame_stats {
    uint32_t splats, visible, pairs, reserved;
    double project_ms, depth_sort_ms, counts_ms, emit_ms, tile_sort_ms, blend_ms, total_ms;
} lrt_frame_stats;

/* RenderTargets (TileRasterizer.h:128-134): caller-owned device images,
 * width * height, bottom row first. colour is float4 premultiplied linear,
 * depth is float view z. */
typedef struct lrt_targets {
    uint32_t width, height;
    void* colour;
    void* depth;
} lrt_targets;

/* Device views of one frame's intermediate buffers, for parity checks. Valid
 * until the next call on the handle. */
typedef struct lrt_debug_view {
    const void* proj;            /* 48-byte ProjRecord per slot (frame.slang:85-89) */
    const void* rects;           /* uint32 x4 per slot: tile rect lo.x lo.y hi.x hi.y */
    const void* touched;         /* uint32 per slot */
    const void* depth_keys;      /* uint32 per slot: float bits of view z >> 7; 0x00FFFFFF culled */
    const void* pairs;           /* uint64 per pair, sorted: tile | depth key | slot (see pair_*) */
    const void* ranges;          /* uint32 x2 per tile: [start, end) into pairs */
    uint32_t slots, pairs_count, tiles, slot_bits;
    uint32_t depth_bits, tile_bits, visible, reserved;
} lrt_debug_view;

typedef struct lrt_rast lrt_rast;

uint32_t lrt_abi_version(void);

/* TileRasterizer::create. `device` is the CUDA ordinal the handle renders on. */
int lrt_rast_create(lrt_rast** out, int device);
void lrt_rast_destroy(lrt_rast* rast);
/* The message of the last failed call on this handle ("" when none). */
const char* lrt_rast_last_error(const lrt_rast* rast);

/* TileRasterizer::render(const Projection&, instances, settings, targets).
 * `stream` is a cudaStream_t (NULL: the legacy default stream). Instances are
 * concatenated into slots base + i in the order given; the slot breaks depth
 * ties. Like the reference's render (which ends with a blocking submit) the
 * call returns when the frame is done; it reads back the counts and the
 * device status once, at the end. A frame (or view) side above 2^19 pixels
 * returns LRT_UNSUPPORTED, as do more than 2^32 splats or pairs. */
int lrt_rast_render(lrt_rast* rast, const lrt_projection* projection,
                    const lrt_splat_instance* instances, uint32_t instance_count,
                    const lrt_render_settings* settings, lrt_targets* targets,
                    lrt_frame_stats* stats, void* stream);

/* The same frame, returning once it is enqueued on `stream`, so the host can
 * prepare the next frame (or read back the last one) while the device
 * renders. No reference counterpart: the reference's render always ends with
 * a blocking submit. A frame is only enqueued when a frame of the same shape
 * (splat count, width, height) has run with lrt_rast_render or this call's
 * waiting path and the last pair count read leaves a quarter of the pair
 * buffer free; otherwise this call waits like lrt_rast_render (a frame of
 * a known shape that leaves less free first grows the buffer, so that the
 * frames after it are enqueued again). time_stages also makes it wait. Enqueued frames are ordered after every earlier call on
 * the handle, on any stream; targets belong to the caller until the frame is
 * done (an event the caller records on `stream` after this call marks it).
 * Counts and device status of enqueued frames are read by lrt_rast_settle. */
/* TileRasterizer::render with its `points` and `under` arguments
 * (TileRasterizer.cpp:188-484): the point instances are projected as opaque
 * discs into slots after the splats and sorted with them, and `under` (may be
 * NULL; the frame's size, linear premultiplied colour and view depth, bottom
 * row first) is a layer the splats composite over: a pixel stops at the
 * first pair at or behind the layer's depth there, or at the first disc it
 * touches, and what stopped it shows through the remaining transmittance
 * (shaders/lrt/splat/splat_blend.slang:23-120, splatBlendComposite). With no
 * points and no layer it is lrt_rast_render. */
int lrt_rast_render_composite(lrt_rast* rast, const lrt_projection* projection,
                              const lrt_splat_instance* instances, uint32_t instance_count,
                              const lrt_point_instance* points, uint32_t point_count,
                              const lrt_targets* under, const lrt_render_settings* settings,
                              lrt_targets* targets, lrt_frame_stats* stats, void* stream);

int lrt_rast_render_async(lrt_rast* rast, const lrt_projection* projection,
                          const lrt_splat_instance* instances, uint32_t instance_count,
                          const lrt_render_settings* settings, lrt_targets* targets, void* stream);

/* Waits for every enqueued frame. Returns LRT_OVERFLOW when any of them
 * emitted more pairs than the buffer held (their images are incomplete; the
 * buffers are grown, so drawing them again succeeds), LRT_TIMEOUT when a
 * bounded device wait gave up, else LRT_OK. `stats` (may be NULL) receives
 * the splats, visible splats and pairs of the last frame. */
int lrt_rast_settle(lrt_rast* rast, lrt_frame_stats* stats);

int lrt_rast_debug_view(lrt_rast* rast, lrt_debug_view* out);

/* One view of a batch: its projection, size and caller-owned device images
 * (colour float4 and depth float, width * height, bottom row first). */
typedef struct lrt_view {
    lrt_projection projection;
    uint32_t width, height;
    void* colour;
    void* depth;
} lrt_view;

/* How a batch was run: views per chunk (each chunk is one projection pass,
 * one sort and one persistent blend launch) and blend blocks per SM, chosen
 * by the autotuner on the first batch of a given shape; whether the chunks
 * were replayed from a captured CUDA graph. */
typedef struct lrt_batch_stats {
    uint32_t views, splats, pairs, chunks;
    uint32_t views_per_chunk, blend_blocks_per_sm, graph_replayed, reserved;
    double device_ms;   /* CUDA-event time of the batch on the device */
    double total_ms;    /* host wall time of the call */
} lrt_batch_stats;

/* Many views of the same instances in one call (no reference counterpart:
 * the reference renders one view per call). Every view is the frame
 * lrt_rast_render would draw -- the same pixels, bit for bit -- with the
 * settings' width and height replaced by the view's. Each chunk of views is
 * projected view by view into one pair buffer whose tile ids number the
 * chunk's tiles one view after another, sorted once, and blended by one
 * persistent launch that takes (view, tile) work items from a queue. The
 * first batch of a given shape (view count and sizes, splat count) is timed
 * under a few chunk sizes and blend grid sizes and the fastest kept; the
 * next one is captured into a CUDA graph, and later ones replay it with the
 * new cameras. Returns when the batch is done. */
int lrt_rast_render_batch(lrt_rast* rast, const lrt_splat_instance* instances, uint32_t instance_count,
                          const lrt_view* views, uint32_t view_count, const lrt_render_settings* settings,
                          lrt_batch_stats* stats, void* stream);

/* Camera::lookingAt and projectionFor, in double precision on the host. */
int lrt_camera_looking_at(const double eye[3], const double target[3], const double up[3],
                          lrt_camera* out);
int lrt_projection_for(const lrt_camera* camera, uint32_t width, uint32_t height,
                       lrt_projection* out);

/* Differentiable parameters of one cloud for the training path (device
 * pointers; fp32 unless noted): means [n][3], log_scales [n][3], quats [n][4]
 * as (w, x, y, z), normalised in the forward (16-byte aligned),
 * opacity_logits [n], sh [n][16][3] fp16 (DC first, then the 15 rest
 * coefficients, rgb per basis; 16-byte aligned). The forward is the plain
 * forward with scale exp(log_scale), opacity sigmoid(logit) and base colour
 * 0.5 + SH0 * DC, without the packed layout's quantisation. No reference
 * counterpart: the reference renders only.
 *
 * flags: LRT_TRAIN_SORT_VALUES carries each pair's emit index (what the
 * backward pass indexes its per-pair partials by) through the pair sort as a
 * 32-bit value. By default it is the pair word's low field instead, with a
 * 4-byte emit-index -> slot map the blend reads, which makes the sort move
 * 8 bytes per pair, not 12; the value form is chosen by itself when tile,
 * depth key and emit index do not fit 64 bits (beyond 2^(40 - tile bits)
 * pairs). Both give the same images and gradients. */
#define LRT_TRAIN_SORT_VALUES 1u
typedef struct lrt_train_params {
    uint32_t count;
    uint32_t flags;
    const void* means;
    const void* log_scales;
    const void* quats;
    const void* opacity_logits;
    const void* sh;
} lrt_train_params;

/* Gradients of the same shapes (fp32 throughout; the SH gradient is fp32
 * over the fp16 coefficients, 16-byte aligned). Written, not accumulated. */
typedef struct lrt_train_grads {
    void* means;
    void* log_scales;
    void* quats;
    void* opacity_logits;
    void* sh;
} lrt_train_grads;

/* The training forward: renders `params` (one cloud in world space) like
 * lrt_rast_render and keeps on the handle what lrt_rast_train_backward needs.
 * The parameter buffers must stay unchanged until the backward. The first
 * call on a handle waits for its frame (sizing the pair buffers, drawing
 * again if they were short); later calls only enqueue it (unless
 * settings->time_stages is set), so the caller's loss and the backward can be
 * queued behind it, and the stats then carry only the splat count. Such a
 * frame's counts and status are checked by lrt_rast_train_backward, which
 * returns LRT_OVERFLOW (buffers grown; run the step again) if the frame
 * emitted more pairs than the buffers held. */
int lrt_rast_train_forward(lrt_rast* rast, const lrt_projection* projection, const lrt_train_params* params,
                           const lrt_render_settings* settings, lrt_targets* targets, lrt_frame_stats* stats,
                           void* stream);
/* The backward of the last lrt_rast_train_forward on this handle (no other
 * render in between): grad_colour is dL/d(colour) as float4 [height][width]
 * (device); gradients of the parameters are written to `grads`. A
 * reverse-order re-blend per pixel, per-pair partials written at each pair's
 * emit index, then a per-splat ordered sum and the projection's chain rule:
 * no atomics. It enqueues its kernels on `stream` (the gradients are ready
 * in that stream's order), then, after a forward that was only enqueued,
 * waits for that forward's counts: if that frame emitted more pairs than the
 * buffers held it returns LRT_OVERFLOW and the gradients it wrote are not to
 * be used (run the step again; the buffers are grown). */
int lrt_rast_train_backward(lrt_rast* rast, const void* grad_colour, lrt_train_grads* grads, void* stream);
/* CUDA-event times of the last backward: the blend backward and the
 * per-splat reduction + projection backward (waits for the backward). */
int lrt_rast_backward_times(const lrt_rast* rast, double* blend_ms, double* project_ms);

/* One view of a training batch: a batch view (its images written by the
 * forward) plus the loss's target image, float3 per pixel (width * height,
 * bottom row first), and where its loss goes (a device float; may be NULL). */
typedef struct lrt_train_view {
    lrt_projection projection;
    uint32_t width, height;
    void* colour;
    void* depth;
    const void* target;
    void* loss;
} lrt_train_view;

/* A training step over many views of one cloud of raw parameters, in one
 * call (no reference counterpart): for each view, the forward of
 * lrt_rast_train_forward (its colour and depth written, the same pixels bit
 * for bit), the L1 loss of lrt_rast_l1_loss against the view's target, and
 * the backward of that loss; `grads` receives the gradients of the sum of the
 * views' losses (written, not added to), accumulated view by view in the
 * given order, so they are the sum of the single-view gradients taken in that
 * order, bit for bit (up to the sign of a zero). Views go in chunks: each
 * chunk is projected view by view into one pair buffer (the views' tiles
 * numbered one after another), sorted once, blended by one persistent launch
 * over (view, tile) items, and taken back through one backward-blend launch
 * over those items and one per-splat backward over the chunk's views (each
 * splat's view gradients summed in order, its gradient buffers written once
 * a chunk). The settings' width and height are replaced
 * by each view's. Returns when the step is done; OVERFLOW cannot happen (a
 * chunk whose pairs outgrow their buffer is drawn again with more room). */
int lrt_rast_train_batch(lrt_rast* rast, const lrt_train_params* params, const lrt_train_view* views,
                         uint32_t view_count, const lrt_render_settings* settings, lrt_train_grads* grads,
                         lrt_batch_stats* stats, void* stream);

/* Test hook of lrt_rast_train_batch (no counterpart in the reference): fixes
 * its views per chunk and blend blocks per SM for the handle's later steps
 * instead of timing candidates (0, 0: tune again). */
int lrt_rast_debug_train_chunking(lrt_rast* rast, uint32_t views_per_chunk, uint32_t blocks_per_sm);


/* PrefixSum::apply: exclusive scan of `count` uint32 at `in` into `out`, the
 * sum into `total` (all device pointers; `out` may alias `in`). Single pass,
 * decoupled look-back; scratch is the handle's. */
int lrt_prefix_sum(lrt_rast* rast, const void* in, void* out, void* total, uint32_t count,
                   void* stream);

/* RadixSort::sort: stable LSD sort of `count` keys (key_bytes 4 or 8) and
 * optional uint32 values by their low `key_bits` bits, in place. Onesweep:
 * one histogram pass, then one decoupled look-back pass per 8-bit digit. */
int lrt_radix_sort(lrt_rast* rast, void* keys, void* values, uint32_t count, uint32_t key_bits,
                   uint32_t key_bytes, void* stream);

/* The Mip-Splatting 3D filter's per-splat variance (Yu et al., CVPR 2024,
 * section 4.1), from a set of cameras: a splat's sampling rate under a
 * camera is focal_x / z (perspective; focal_x for an orthographic camera)
 * where its centre lies in front of the near plane and projects within the
 * image widened by 15% on each side; its variance is coefficient / r^2 with r
 * the highest such rate (the paper's default coefficient is 0.2). Splats no
 * camera sees get the largest variance among the seen ones; with none seen,
 * 0. `cloud` and `variance` are device memory; cameras and sizes (width,
 * height per camera) are host arrays; positions are taken in the cloud's
 * own space (cameras given in that space). No counterpart in the reference. */
int lrt_rast_filter3d(lrt_rast* rast, const lrt_gpu_splats* cloud, const lrt_projection* cameras,
                      const uint32_t* sizes, uint32_t camera_count, float coefficient, float* variance,
                      void* stream);

/* Test hooks of a handle's lrt_radix_sort (no counterpart in the reference,
 * whose sort never waits on another workgroup):
 *   skip_first_partition  the last digit pass runs with partition 0 never
 *       taken, so the partition after it waits for counts nobody publishes.
 *       That wait gives up after `poll_limit` polls (0: the normal limit,
 *       2^22), the call returns LRT_TIMEOUT, and the keys are left in an
 *       undefined order (every write stays inside the buffers);
 *   wide_look_back  the 64-bit look-back words that sorts of 2^30 keys or
 *       more use, at any size.
 * Clearing them (0, 0, 0) restores normal sorts; the handle stays usable
 * throughout. */
int lrt_rast_debug_sort(lrt_rast* rast, uint32_t skip_first_partition, uint32_t poll_limit,
                        uint32_t wide_look_back);

/* The prefix sum above for callers that cannot allocate device memory: a
 * plugin running inside a host application that owns every device allocation
 * (and its budget), or a frame-critical path where cudaMalloc would
 * synchronise the device. It takes no handle and allocates nothing: the
 * caller passes input, output and total (device pointers), and the scan's
 * look-back scratch is a fixed 128 KB array compiled into the library, which
 * every GPU that loads the library holds until the process exits. Counts
 * above LRT_PREFIX_SUM_NOALLOC_MAX are rejected with LRT_INVALID_ARGUMENT.
 * The first call on each device looks up that array's device address (with
 * the device current).
 * All calls on a device share the array and clear it on their stream first;
 * calls whose work overlaps on the GPU race on it. Blocks until done, like
 * lrt_prefix_sum. No counterpart in the reference: its PrefixSum always
 * allocates through its device. */
#define LRT_PREFIX_SUM_NOALLOC_MAX (1u << 26)
int lrt_prefix_sum_noalloc(const void* in, void* out, void* total, uint32_t count, void* stream);

/* Raw 3DGS records (the PLY encoding: x y z, logit opacity, 3 log scales,
 * rot w x y z, 3 DC, rest coefficients all red then green then blue) to the
 * packed layout above, on the host. Invalid records (non-finite position or
 * scale, |log scale| >= 60, opacity < 1/255) are dropped, order kept. Writes
 * positions (float4), shape (uint32 x4) and sh (sh_words uint32; one word
 * minimum per splat) for up to `count` splats; returns the kept count in
 * *kept. `keep_per_colour` <= `file_per_colour` (0, 3, 8, 15). */
int lrt_pack_splats(const float* raw, uint32_t count, uint32_t floats_per_record,
                    uint32_t file_per_colour, uint32_t keep_per_colour, float* positions,
                    uint32_t* shape, uint32_t* sh, uint32_t* kept);

/* io::SplatEncoding (io/RawSplats.h:15-70): where a raw record's fields are,
 * in floats from its start, and how each is encoded. Modes:
 *   opacity_mode  0 logit, 1 linear, 2 byte (v / 255)
 *   scale_mode    0 log, 1 linear, 2 SPZ byte (log scale = v / 16 - 10)
 *   colour_mode   0 SH DC (0.5 + SH0 v), 1 linear, 2 byte, 3 SPZ byte,
 *                 4 linear light (taken to the sRGB curve the blend undoes)
 *   rotation_mode 0 floats w x y z, 1 bytes ((v - 128) / 128),
 *                 2 SPZ first three (x y z bytes, w from unit length),
 *                 3 SPZ smallest three (a uint32 in two 16-bit halves at
 *                 rot_x and rot_y)
 *   rest_mode     0 floats, 1 bytes ((v - 128) / 128)
 * rest_colour_outer 1: the rest coefficients are all red, then green, then
 * blue (3DGS PLY), 0: rgb per basis (SPZ). flip_yz: the file is right-up-
 * back, and y and z of positions, rotations and harmonics change sign.
 * lrt_splat_encoding_ply fills the 3DGS PLY layout. */
typedef struct lrt_splat_encoding {
    uint32_t floats_per_record;
    uint32_t x, y, z, opacity;
    uint32_t scale0, scale1, scale2;
    uint32_t rot_w, rot_x, rot_y, rot_z;
    uint32_t dc0, dc1, dc2;
    uint32_t rest_base, rest_per_colour, rest_colour_outer;
    uint32_t opacity_mode, scale_mode, colour_mode, rotation_mode, rest_mode;
    float position_scale;
    uint32_t flip_yz;
} lrt_splat_encoding;

int lrt_splat_encoding_ply(uint32_t rest_per_colour, lrt_splat_encoding* out);

/* CloudLoader::upload's decode on the device (GpuClouds.cpp:151-226,
 * splat_validate.slang, splat_decode.slang): `count` raw records (a device
 * pointer, floats_per_record floats each) are validated (finite position and
 * log scales under 60 in size, opacity at least 1/255), compacted in order
 * and packed into the caller's device buffers of `count` capacity
 * (positions float4, shape uint32 x4, sh (keep_per_colour * 3 + 1) / 2 words,
 * one minimum), in one kernel. Returns the kept count in *kept (the call
 * waits for it). keep_per_colour <= rest_per_colour. The per-splat material
 * words of converted meshes (relighting) are not produced. */
int lrt_rast_decode_splats(lrt_rast* rast, const void* raw, uint32_t count, const lrt_splat_encoding* encoding,
                           uint32_t keep_per_colour, void* positions, void* shape, void* sh, uint32_t* kept,
                           void* stream);

/* The same for points (points_validate.slang, points_decode.slang): `count`
 * raw x y z r g b records on the device into positions and colours, as
 * lrt_pack_points does on the host. */
int lrt_rast_decode_points(lrt_rast* rast, const void* raw, uint32_t count, uint32_t colour_kind, float detail,
                           void* positions, void* colours, uint32_t* kept, void* stream);

/* ImageDifference and HdrDifference (ReferenceRenderer.h:50-64). */
typedef struct lrt_image_difference {
    uint64_t pixels;
    uint32_t p99;        /* 99th percentile of the per-pixel largest code difference */
    uint32_t max;
    uint64_t over2;      /* pixels differing by more than 2 code values */
} lrt_image_difference;

typedef struct lrt_hdr_difference {
    uint64_t pixels;
    double rel_mse;      /* mean over pixels of the channel mean (a - b)^2 / (b^2 + 1e-2) */
    double p99_relative; /* 99th percentile of max_c |a - b| / max(|b|, 1e-3), to 9% */
    double max_relative;
} lrt_hdr_difference;

/* compareImages (ReferenceRenderer.cpp:248-297) on the device: two float4
 * images (device pointers, linear premultiplied) in 8-bit sRGB code values.
 * `histogram` (may be NULL) receives the 256 bins on the host. */
int lrt_rast_compare_images(lrt_rast* rast, const void* a, const void* b, uint32_t width, uint32_t height,
                            lrt_image_difference* out, uint32_t* histogram, void* stream);

/* compareHdr (ReferenceRenderer.cpp:299-362) on the device. */
int lrt_rast_compare_hdr(lrt_rast* rast, const void* a, const void* b, uint32_t width, uint32_t height,
                         lrt_hdr_difference* out, void* stream);

/* countDifferent (ReferenceRenderer.cpp:364-396): differing entries of two
 * uint32 device buffers. */
int lrt_rast_count_different(lrt_rast* rast, const void* a, const void* b, uint32_t count, uint64_t* out,
                             void* stream);

/* The photometric L1 loss of a training step (no reference counterpart):
 * mean |colour.rgb - target| over `pixels` pixels and 3 channels, colour a
 * float4 image and target a float3 image (device pointers), written to the
 * device float *loss, summed in a fixed order. Enqueued only. */
int lrt_rast_l1_loss(lrt_rast* rast, const void* colour, const void* target, uint32_t pixels, void* loss,
                     void* stream);

/* Its gradient: grad_colour (float4 per pixel) = sign(colour.rgb - target)
 * / (3 pixels) scaled by *grad_loss (a device float; NULL: 1), alpha 0. */
int lrt_l1_loss_grad(const void* colour, const void* target, uint32_t pixels, const void* grad_loss,
                     void* grad_colour, void* stream);

/* Raw point records (x y z r g b, 6 floats) to the GpuPoints layout above, on
 * the host (the upload half of CloudLoader for points: points_validate.slang
 * and points_decode.slang). colour_kind: 0 none (white), 1 sRGB bytes in
 * 0..255, 2 linear floats. Points with a non-finite position are dropped,
 * and with detail < 1 only those whose index hash falls below it are kept,
 * order kept. Writes up to `count` points; the kept count in *kept. */
int lrt_pack_points(const float* raw, uint32_t count, uint32_t colour_kind, float detail,
                    float* positions, uint32_t* colours, uint32_t* kept);

/* ---- Levels of detail (modules/lod/include/lrt/lod/Lod.h) ----------------
 * A cloud's octree levels of detail, built and cut on the device. The method
 * is the reference's (shaders/lrt/lod/lod_common.slang:1-33): splats in
 * Morton order; per octree cell the additive moments of its splats turned
 * back into one Gaussian; per frame, a cell is drawn merged when it projects
 * to at most `threshold` pixels and its parent does not, a splat when its
 * finest merged cell does not. In memory only: every chunk of splats is
 * resident (the .lrtc streaming store is not provided). */

/* LodBuildSettings (Lod.h:83-93). */
typedef struct lrt_lod_build_settings {
    float max_group_fraction;   /* 0.5: the finest stored level is the deepest whose groups
                                   number at most this fraction of the splats */
    uint32_t coarsest_level;    /* 1 (clamped to 1..10) */
    uint32_t chunk_splats;      /* 65536: splats per chunk, reported only */
    uint32_t reserved;
} lrt_lod_build_settings;

int lrt_lod_build_settings_default(lrt_lod_build_settings* out);

/* LodCloud (Lod.h:41-80): library-owned device buffers. */
typedef struct lrt_lod lrt_lod;

typedef struct lrt_lod_info {
    uint32_t count;             /* splats */
    uint32_t rest_per_colour, sh_words;
    uint32_t levels;            /* stored merged levels, consecutive octree levels */
    uint32_t coarsest, finest;  /* their octree levels */
    uint32_t merged;            /* merged Gaussians over all stored levels */
    uint32_t chunk_splats;
    float bounds_lo[3], bounds_hi[3];
    float extent;               /* the bounds' largest edge (x 1.0001): cells are cubes */
    uint32_t level_groups[10];  /* per stored level, coarsest first */
} lrt_lod_info;

/* LodBuilder::build (Lod.cpp:86-300). `cloud` holds device pointers in the
 * packed layout (rest_per_colour 0, 3, 8 or 15; sh_words at least
 * (rest_per_colour * 3 + 1) / 2, and the merged levels' rows take as many
 * words, zero past the coefficients); `bounds` (host, may be NULL:
 * computed from the positions) is lo xyz then hi xyz; `settings` may be NULL
 * (the defaults). The cloud is not changed; the result owns a Morton-ordered
 * copy. Waits for the build. An empty cloud is LRT_INVALID_ARGUMENT. */
int lrt_lod_build(lrt_rast* rast, const lrt_gpu_splats* cloud, const float* bounds,
                  const lrt_lod_build_settings* settings, lrt_lod** out, void* stream);
void lrt_lod_destroy(lrt_lod* lod);
int lrt_lod_get_info(const lrt_lod* lod, lrt_lod_info* out);

/* The Morton-ordered splats (LodCloud::splats) and each one's 30-bit code. */
int lrt_lod_splats(const lrt_lod* lod, lrt_gpu_splats* out, const uint32_t** codes);

/* Stored level `index` (0 = coarsest): its octree level, its merged Gaussians
 * (LodLevel::gaussians) and per Gaussian its cell code (LodLevel::cells). */
int lrt_lod_level(const lrt_lod* lod, uint32_t index, uint32_t* level, lrt_gpu_splats* gaussians,
                  const uint32_t** cells);

/* The finest stored level's groups' first splats (LodCloud::starts). */
int lrt_lod_starts(const lrt_lod* lod, const uint32_t** starts, uint32_t* groups);

/* LodInstance (Lod.h:106-111). threshold < 0: the call's. */
typedef struct lrt_lod_instance {
    const lrt_lod* cloud;
    double object_to_world[16];
    lrt_splat_edit edit;
    float threshold;
    uint32_t reserved;
} lrt_lod_instance;

/* CutStats (Lod.h:113-124) without the streaming needs. */
typedef struct lrt_cut_stats {
    uint32_t splats;      /* the cloud's own splats drawn */
    uint32_t merged;      /* merged Gaussians drawn */
    uint32_t available;   /* splats in the cloud */
    uint32_t reserved;
} lrt_cut_stats;

/* CutSelector::select (Lod.cpp:349-547): each instance's cut for this view
 * as instances the rasteriser draws. out receives up to `count` instances
 * (those drawing anything, in order; *out_count of them); their clouds belong
 * to `rast` and are rewritten by its next lrt_lod_select. stats (may be NULL)
 * receives one entry per instance. The drawn cloud lists the merged
 * Gaussians, coarsest level first, then the splats, in Morton order. One
 * kernel per instance and one wait for all of them. */
int lrt_lod_select(lrt_rast* rast, const lrt_projection* projection, const lrt_lod_instance* instances,
                   uint32_t count, float threshold, lrt_splat_instance* out, uint32_t* out_count,
                   lrt_cut_stats* stats, void* stream);

/* Diagnostic: the library's own exp (fn 0), log (1), sRGB-to-linear (2),
 * cut-off power (3), float-to-half rounding (4, the binary16 bits in the
 * low 16 bits of each output word) and the half-pair packing of x and -x/2
 * (5, x in the low half) and the blend's exp without range checks (6,
 * defined for -87 <= x <= 88), evaluated on the device over n floats (device pointers),
 * for comparing their bits with a host implementation. No reference
 * counterpart: the reference evaluates these through Slang's library. */
int lrt_math_eval(int fn, const void* x, void* y, uint32_t n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LRT_RASTER_H */
