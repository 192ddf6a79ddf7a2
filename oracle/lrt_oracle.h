/*
 * ORACLE -- test infrastructure, not product code.
 *
 * A CPU restatement of lucabRTrender's splat tile rasteriser, written from the
 * reference's Slang kernels and host code (paths inside the lucabRTrender
 * tree; each function in lrt_oracle.cpp cites the lines it follows). Only the
 * tests, the smoke check and the benchmark's CPU-baseline leg load it, and
 * only to check or time against. The product never calls it.
 *
 * Pinning: the reference's kernels are Slang, compiled at run time through
 * slang-rhi; neither is available here, so the restatement cannot be run
 * against the Slang itself. It is pinned by (1) the reference's own
 * known-answer tests (tests/render/test_splat_render.cpp, tests/scene/
 * test_loading.cpp, tests/gpu/test_algo.cpp), restated as Python tests, and
 * (2) golden camera vectors produced by the reference's own C++ camera code
 * (modules/render/src/Camera.cpp) compiled from its sources under oracle/_ref.
 * Bit-level behaviour of Slang's exp/log/pow lowering is unpinned; this
 * restatement uses its own exp/log (see lrt_oracle.cpp) with the same method
 * the product uses, so the product is checked bit for bit against it.
 */
#ifndef LRT_ORACLE_H
#define LRT_ORACLE_H

#include "../include/lrt_raster.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Host-pointer outputs of one frame, each optional (NULL: not written). */
typedef struct ora_frame_out {
    float* colour;        /* width*height float4 */
    float* depth;         /* width*height */
    float* proj;          /* slots x 12 floats (ProjRecord) */
    uint32_t* rects;      /* slots x 4 */
    uint32_t* touched;    /* slots */
    uint32_t* depth_keys; /* slots */
    uint32_t* pair_tiles; /* pairs, sorted */
    uint32_t* pair_slots; /* pairs, sorted */
    uint32_t* ranges;     /* tiles x 2 */
    uint64_t pair_capacity;
    /* filled in */
    uint64_t pairs;
    uint32_t visible;
    uint32_t slots;
    double stage_ms[6];   /* project, depth sort, counts, emit, tile sort+ranges, blend */
    /* optional: one byte per tile; when set, only tiles with a nonzero byte
       are blended (the other pixels are left as the caller filled them) */
    const uint8_t* blend_tiles;
} ora_frame_out;

uint32_t ora_abi_version(void);
float ora_exp(float x);
float ora_log(float x);
float ora_pow(float x, float y);
void ora_math_eval(int fn, const float* x, float* y, uint32_t n);
uint16_t ora_f32_to_f16(float f);
float ora_f16_to_f32(uint16_t h);

int ora_camera_looking_at(const double eye[3], const double target[3], const double up[3],
                          lrt_camera* out);
int ora_projection_for(const lrt_camera* camera, uint32_t width, uint32_t height,
                       lrt_projection* out);

int ora_pack_splats(const float* raw, uint32_t count, uint32_t floats_per_record,
                    uint32_t file_per_colour, uint32_t keep_per_colour, float* positions,
                    uint32_t* shape, uint32_t* sh, uint32_t* kept);

/* The Mip-Splatting 3D filter's variance per splat (lrt_rast_filter3d's
 * definition; host pointers). */
int ora_filter3d(const lrt_gpu_splats* cloud, const lrt_projection* cameras, const uint32_t* sizes,
                 uint32_t camera_count, float coefficient, float* variance);

/* The tile rasteriser (splats in lrt_gpu_splats are HOST pointers here). */
int ora_render(const lrt_projection* projection, const lrt_splat_instance* instances,
               uint32_t instance_count, const lrt_render_settings* settings,
               ora_frame_out* out, uint32_t threads);

/* The training path's forward: one cloud of raw parameters (HOST pointers,
 * layout of lrt_train_params) in world space, rendered like ora_render. For
 * each pixel of the crop, the slots that contribute to it, in blend order,
 * are written to list_slots; pixel k's list is
 * [list_offsets[k], list_offsets[k + 1]). */
int ora_train_render(const lrt_projection* projection, const lrt_train_params* params,
                     const lrt_render_settings* settings, ora_frame_out* out, uint32_t threads, uint32_t crop_x0,
                     uint32_t crop_y0, uint32_t crop_w, uint32_t crop_h, uint32_t* list_offsets,
                     uint32_t* list_slots, uint64_t list_capacity, uint64_t* list_total);

/* The rasteriser with point instances drawn as opaque discs and an optional
 * under layer (TileRasterizer::render's `points` and `under`,
 * splatBlendComposite). Points and the under layer are HOST pointers;
 * under_colour / under_depth may be NULL. */
int ora_render_composite(const lrt_projection* projection, const lrt_splat_instance* instances,
                         uint32_t instance_count, const lrt_point_instance* points, uint32_t point_count,
                         const float* under_colour, const float* under_depth, const lrt_render_settings* settings,
                         ora_frame_out* out, uint32_t threads);

/* The brute force with point discs (ReferenceRenderer::render's `points`). */
int ora_reference_render_composite(const lrt_projection* projection, const lrt_splat_instance* instances,
                                   uint32_t instance_count, const lrt_point_instance* points, uint32_t point_count,
                                   const lrt_render_settings* settings, float* colour, float* depth,
                                   uint32_t* overflow, uint32_t threads);

/* Raw splat records of any encoding to the packed layout (as
 * lrt_rast_decode_splats does on the device), host pointers. */
int ora_decode_splats(const float* raw, uint32_t count, const lrt_splat_encoding* encoding, uint32_t keep,
                      float* positions, uint32_t* shape, uint32_t* sh, uint32_t* kept);

/* Raw point records (x y z r g b) to positions/colours, as lrt_pack_points. */
int ora_pack_points(const float* raw, uint32_t count, uint32_t colour_kind, float detail, float* positions,
                    uint32_t* colours, uint32_t* kept);

/* The reference points test's randomPoints (tests/render/test_points.cpp:22-44). */
int ora_random_points(uint32_t count, uint64_t seed, float* raw);

/* The brute-force ground truth (ReferenceRenderer). Returns the number of
 * pixels whose contributor count passed kMaxHits in *overflow. */
int ora_reference_render(const lrt_projection* projection, const lrt_splat_instance* instances,
                         uint32_t instance_count, const lrt_render_settings* settings,
                         float* colour, float* depth, uint32_t* overflow, uint32_t threads);

/* compareImages: 8-bit sRGB code difference histogram of two float4 images. */
int ora_compare_images(const float* a, const float* b, uint32_t width, uint32_t height,
                       uint32_t* histogram256, uint32_t* p99, uint32_t* max, uint64_t* over2,
                       uint64_t* pixels);

/* compareHdr's histogram and relative squared error (the device's order). */
int ora_compare_hdr(const float* a, const float* b, uint32_t width, uint32_t height, uint32_t* histogram256,
                    float* error);
uint64_t ora_count_different(const uint32_t* a, const uint32_t* b, uint32_t count);

/* The reference test fixture's randomCloud (tests/render/SplatFixtures.h:48-85):
 * `count` degree-1 raw records of 23 floats. */
int ora_random_cloud(uint32_t count, uint64_t seed, float min_size, float max_size,
                     float min_opacity, float max_opacity, float* raw);

/* Levels of detail (LodBuilder::build, CutSelector::select), host pointers
 * in `cloud`. Built in the reference's own schedule: a stable sort, one
 * boundary pass and prefix sum per level, merges through the per-splat group
 * index. ora_lod_describe fills an lrt_lod_info (chunk_splats 0). */
typedef struct ora_lod ora_lod;
int ora_lod_build(const lrt_gpu_splats* cloud, const float* bounds, float max_group_fraction,
                  uint32_t coarsest_level, ora_lod** out);
void ora_lod_free(ora_lod* lod);
int ora_lod_describe(const ora_lod* lod, lrt_lod_info* out);
/* which: 0 store positions, 1 store shape, 2 store sh, 3 codes, 4 finest
 * starts, 5 merged positions, 6 merged shape, 7 merged sh, 8 cells (all
 * levels, coarsest first). */
int ora_lod_copy(const ora_lod* lod, int which, void* dst);
/* One instance's cut; the outputs hold the cloud's splat count. */
int ora_lod_cut(const ora_lod* lod, const lrt_projection* projection, const double object_to_world[16],
                float threshold, float* positions, uint32_t* shape, uint32_t* sh, uint32_t* splats,
                uint32_t* merged);

#ifdef __cplusplus
}
#endif

#endif
